/* rt_b200_host.h -- host-side domains, extremal tilings, height functions and
 * conversions of librt_b200.so (no GPU needed).
 *
 * These replace the static helpers of the reference's Tiler classes.  Every
 * function writes a variable-length int32 array: *len receives the length;
 * the array is written when out != NULL and cap >= *len (out == NULL is a
 * size query; where the length follows from the input sizes -- extremal
 * tilings, heights, vertex kinds -- the query computes nothing else, so
 * checks of the domain itself come with the call that fills the array).  Domains, tilings and height functions use the reference's
 * encodings and sizes, so outputs are interchangeable with it.  Heights are
 * normalised as the reference does: 0 at the first boundary vertex in
 * row-major order, INT_MAX outside the domain.  A domain that is not
 * tileable returns RT_E_INVAL (the reference prints a message and returns a
 * partial result).
 */
#ifndef RT_B200_HOST_H
#define RT_B200_HOST_H

#include <stdint.h>

#include "rt_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- dominoes (src/Domino/DominoTiler.h:83-107) ---- */
/* DominoTiler::Rectangle(M, N), src/Domino/DominoTiler.cpp:118-129 */
rt_status rt_domino_rectangle(int32_t rows, int32_t cols, int32_t* out, int64_t cap, int64_t* len);
/* DominoTiler::AztecRectangle(N, remove), src/Domino/DominoTiler.cpp:136-193 */
rt_status rt_domino_aztec_rectangle(int32_t order, const int32_t* remove, int32_t k, int32_t* out, int64_t cap,
                                    int64_t* len);
/* DominoTiler::AztecDiamond(N), src/Domino/DominoTiler.cpp:131-134 */
rt_status rt_domino_aztec(int32_t order, int32_t* out, int64_t cap, int64_t* len);
/* DominoTiler::DomainToVertices, src/Domino/DominoTiler.cpp:479-499 */
rt_status rt_domino_domain_to_vertices(const int32_t* d, int64_t dlen, int32_t* out, int64_t cap, int64_t* len);
/* DominoTiler::MaxTiling / MinTiling (Thurston), src/Domino/DominoTiler.cpp:214-400 */
rt_status rt_domino_max_tiling(const int32_t* d, int64_t dlen, int32_t* out, int64_t cap, int64_t* len);
rt_status rt_domino_min_tiling(const int32_t* d, int64_t dlen, int32_t* out, int64_t cap, int64_t* len);
/* DominoTiler::HeightfuncToTiling, src/Domino/DominoTiler.cpp:402-421 */
rt_status rt_domino_height_to_tiling(const int32_t* h, int64_t hlen, const int32_t* d, int64_t dlen, int32_t* out,
                                     int64_t cap, int64_t* len);
/* DominoTiler::TilingToHeightfunc, src/Domino/DominoTiler.cpp:423-461 */
rt_status rt_domino_tiling_to_height(const int32_t* t, int64_t tlen, const int32_t* d, int64_t dlen, int32_t* out,
                                     int64_t cap, int64_t* len);
/* DominoTiler::TilingToDomain, src/Domino/DominoTiler.cpp:463-477 */
rt_status rt_domino_tiling_to_domain(const int32_t* t, int64_t tlen, int32_t* out, int64_t cap, int64_t* len);

/* ---- lozenges (src/Lozenge/LozengeTiler.h:61-78) ---- */
/* LozengeTiler::AlmostHexDomain(N, M), src/Lozenge/LozengeTiler.cpp:344-389 */
rt_status rt_lozenge_almost_hex(int32_t side, int32_t cut, int32_t* out, int64_t cap, int64_t* len);
/* Hexagon with sides a, b, c, a, b, c (generalises AlmostHexDomain(N, 0),
 * which is a = b = c = N).  No reference counterpart. */
rt_status rt_lozenge_hexagon(int32_t a, int32_t b, int32_t c, int32_t* out, int64_t cap, int64_t* len);
/* LozengeTiler::DomainToVertices, src/Lozenge/LozengeTiler.cpp:405-434 */
rt_status rt_lozenge_domain_to_vertices(const int32_t* d, int64_t dlen, int32_t* out, int64_t cap, int64_t* len);
/* LozengeTiler::MaxTiling / MinTiling, src/Lozenge/LozengeTiler.cpp:140-318 */
rt_status rt_lozenge_max_tiling(const int32_t* d, int64_t dlen, int32_t* out, int64_t cap, int64_t* len);
rt_status rt_lozenge_min_tiling(const int32_t* d, int64_t dlen, int32_t* out, int64_t cap, int64_t* len);
/* LozengeTiler::HeightfuncToTiling, src/Lozenge/LozengeTiler.cpp:321-342 */
rt_status rt_lozenge_height_to_tiling(const int32_t* h, int64_t hlen, const int32_t* d, int64_t dlen, int32_t* out,
                                      int64_t cap, int64_t* len);
/* LozengeTiler::TilingToHeightfunc, src/Lozenge/LozengeTiler.cpp:95-138 */
rt_status rt_lozenge_tiling_to_height(const int32_t* t, int64_t tlen, const int32_t* d, int64_t dlen, int32_t* out,
                                      int64_t cap, int64_t* len);
/* LozengeTiler::TilingToDomain, src/Lozenge/LozengeTiler.cpp:436-462 */
rt_status rt_lozenge_tiling_to_domain(const int32_t* t, int64_t tlen, int32_t* out, int64_t cap, int64_t* len);

/* ---- rectangle-triangle (src/RectTriangle/RectTriangleTiler.h:60-66) ---- */
/* RectTriangleTiler::maxHex / minHex, src/RectTriangle/RectTriangleTiler.cpp:401-521 */
rt_status rt_recttri_max_hex(int32_t side, int32_t* out, int64_t cap, int64_t* len);
rt_status rt_recttri_min_hex(int32_t side, int32_t* out, int64_t cap, int64_t* len);
/* RectTriangleTiler::LozengeToRectTriangle, src/RectTriangle/RectTriangleTiler.cpp:523-565 */
rt_status rt_recttri_from_lozenge(const int32_t* tl, int64_t tlen, const int32_t* dl, int64_t dlen, int32_t* out,
                                  int64_t cap, int64_t* len);

/* ---- triangular-lattice dimers (src/TriangleDimer/TriangleDimerTiler.h:182-195) ---- */
/* TriangleDimerTiler::IceCreamCone(N, M), src/TriangleDimer/TriangleDimerTiler.cpp:485-581 */
rt_status rt_tridimer_ice_cream_cone(int32_t side, int32_t cut, int32_t* out, int64_t cap, int64_t* len);
/* No reference counterpart (the reference builds only IceCreamCone): a
 * "bibone" hexagon -- the triangular-lattice vertices (x, y), 0 <= x, y <= 2s,
 * s <= x + y <= 3s (a hexagon of side s edges, 3s(s+1) + 1 vertices: always
 * odd) without its top-left corner (0, s), so that dimers can cover it --
 * with its canonical start: row by row from the top, a row whose count of
 * free vertices is odd pairs one end vertex with the same end of the next
 * row (the right end, unless the row above took that one), and the rest of
 * the row is paired horizontally from the left.  Vertex (x, y) sits at
 * (x + 3, y + 3) of the eSize = 2s + 8 vertex grid, so the tiling is N x N
 * with N = 4s + 16 and the three outer rows and columns the walk needs stay
 * empty.  1 <= side <= 4096. */
rt_status rt_tridimer_hexagon(int32_t side, int32_t* out, int64_t cap, int64_t* len);
/* TriangleDimerTiler::TestButterfly(type), :583-632 */
rt_status rt_tridimer_test_butterfly(int32_t kind, int32_t* out, int64_t cap, int64_t* len);
/* TriangleDimerTiler::TilingToTriangleFlips / TilingToButterflyFlips, :634-709 */
rt_status rt_tridimer_triangle_flips(const int32_t* t, int64_t tlen, int32_t* out, int64_t cap, int64_t* len);
rt_status rt_tridimer_butterfly_flips(const int32_t* t, int64_t tlen, int32_t* out, int64_t cap, int64_t* len);
/* TriangleDimerTiler::TilingToVertices / TilingToDomain, :711-770 */
rt_status rt_tridimer_vertices(const int32_t* t, int64_t tlen, int32_t* out, int64_t cap, int64_t* len);
rt_status rt_tridimer_tiling_to_domain(const int32_t* t, int64_t tlen, int32_t* out, int64_t cap, int64_t* len);
/* TriangleDimerTiler::DimerIndicator(t, c), :20-84 */
rt_status rt_tridimer_dimer_indicator(const int32_t* t, int64_t tlen, int32_t orient, int32_t* out, int64_t cap,
                                      int64_t* len);

#ifdef __cplusplus
}
#endif
#endif /* RT_B200_HOST_H */
