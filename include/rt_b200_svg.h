/* rt_b200_svg.h -- SVG and text output of librt_b200.so (no GPU needed).
 *
 * Byte-for-byte the files the reference's drawing helpers write (same element
 * templates, same default stream number formatting), so pictures and matrix
 * files are interchangeable with it.  All return RT_OK, or RT_E_INVAL for a
 * null argument or a file that cannot be written.  Writers that take an
 * optional domain `d` derive it from the tiling when d is NULL, like the
 * reference's one-argument overloads.
 */
#ifndef RT_B200_SVG_H
#define RT_B200_SVG_H

#include <stdint.h>

#include "rt_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* DominoTiler::DomainToSVG / TilingToSVG / MayaToSVG / DimerToSVG,
 * src/Domino/DominoTiler.cpp:508-681 */
rt_status rt_domino_domain_svg(const int32_t* d, int64_t dlen, const char* filename);
rt_status rt_domino_tiling_svg(const int32_t* t, int64_t tlen, const char* filename);
rt_status rt_domino_maya_svg(const int32_t* t, int64_t tlen, const char* filename);
rt_status rt_domino_dimer_svg(const int32_t* t, int64_t tlen, const int32_t* d, int64_t dlen, const char* filename);

/* LozengeTiler::DomainToSVG / TilingToSVG / DimerToSVG / PrintDomain,
 * src/Lozenge/LozengeTiler.cpp:391-403, 480-613 */
rt_status rt_lozenge_domain_svg(const int32_t* d, int64_t dlen, const char* filename);
rt_status rt_lozenge_tiling_svg(const int32_t* t, int64_t tlen, const char* filename);
rt_status rt_lozenge_dimer_svg(const int32_t* t, int64_t tlen, const int32_t* d, int64_t dlen, const char* filename);
rt_status rt_lozenge_print_domain(const int32_t* d, int64_t dlen, const char* filename);

/* RectTriangleTiler::TilingToSVG (+ TilePicture), src/RectTriangle/RectTriangleTiler.cpp:567-697 */
rt_status rt_recttri_tiling_svg(const int32_t* t, int64_t tlen, const char* filename);

/* TriangleDimerTiler::DomainToSVG / TilingToSVG / DimerToSVG,
 * src/TriangleDimer/TriangleDimerTiler.cpp:772-902 */
rt_status rt_tridimer_domain_svg(const int32_t* d, int64_t dlen, const char* filename);
rt_status rt_tridimer_tiling_svg(const int32_t* t, int64_t tlen, const char* filename);
rt_status rt_tridimer_dimer_svg(const int32_t* t, int64_t tlen, const int32_t* d, int64_t dlen, const char* filename);

/* SaveMatrix(const std::vector<int>&, std::string) and LoadMatrix,
 * src/common/common.cpp:82-161 */
rt_status rt_save_matrix(const int32_t* a, int64_t len, const char* filename);
rt_status rt_load_matrix(const char* filename, int32_t* out, int64_t cap, int64_t* len);

/* Binary matrices (no reference counterpart): any int32 array (tilings,
 * heights, domains) in the smallest of 1, 2, 4, 8, 16 or 32 bits per value
 * that holds its range, with a checksum -- a domino tiling takes 4 bits a
 * value.  The load returns the count in *len (out NULL: size query only) and
 * RT_E_INVAL for a file that is not this format, truncated or corrupted. */
rt_status rt_save_matrix_binary(const int32_t* a, int64_t len, const char* filename);
rt_status rt_load_matrix_binary(const char* filename, int32_t* out, int64_t cap, int64_t* len);

#ifdef __cplusplus
}
#endif
#endif /* RT_B200_SVG_H */
