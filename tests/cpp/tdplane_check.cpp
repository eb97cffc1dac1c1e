// Host check of the triangle-dimer bit-plane ops (csrc/rt_tdplane.cuh)
// against the integer rule (csrc/rt_tridimer.cuh, TriDimerRule), both
// compiled for the host.  Input: the eight m x m state arrays of a tiling
// (H, L, R, U, D, BH, BL, BR; int32, as the oracle splits them).  The chain
// makes `steps` moves of the fast-mode sweep (move s mod 30, the phase
// program of td_step_phases); every site draws a pseudo-random 23-bit k per
// drawing phase.  At each phase the integer rule advances the state, the
// bit-plane ops are applied to the same state, and all eight arrays must
// agree at every site.
//
//   tdplane_check ARRAYS_FILE M STEPS
//   tdplane_check random M ROUNDS   (every phase of the 30 moves on random
//       states of each array's bit width, ROUNDS times; values compared
//       modulo 2^bits, the width the planes keep)
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

namespace rtb {
// Host stand-ins for the walk kernel's argument block and phase-descriptor
// accessors, which the rule's walk-kernel glue names.
struct WalkArgs {
    int n, wpad;
};
inline uint32_t ph_op(uint32_t d) { return d & 0xffu; }
inline uint32_t ph_a(uint32_t d) { return (d >> 8) & 0xffu; }
inline uint32_t ph_b(uint32_t d) { return (d >> 16) & 0xffu; }
}  // namespace rtb

#include "rt_tdplane.cuh"
#include "rt_tridimer.cuh"

using namespace rtb;

namespace {

struct Phase {
    uint32_t op, a, b;
};

// Move mv of a fast-mode sweep (rt_capi.cu: fast_step_phases / td_step_phases).
std::vector<Phase> phases_of(int mv) {
    if (mv < 6) {
        const uint32_t r1 = mv / 2, r2 = mv % 2;
        return {{TD_ROT_LOZ, r1, r2}, {TD_LOZ_FLIPPED, r1, r2}, {TD_LOZ_OTHER, r1, 0},
                {TD_UP_FROM_LOZ, 0, 0}, {TD_TRI_OTHER, 0, 7}};
    }
    if (mv < 12) {
        const uint32_t r1 = (mv - 6) % 3, r2 = (mv - 6) / 3;
        return {{TD_ROT_TRI, r2, r1}, {TD_TRI_FLIPPED, r2, r1}, {TD_TRI_OTHER, r2, 0},
                {TD_LOZ_FROM_TRI, 0, 0}, {TD_BFLY_FROM_LOZ, 0, 7}};
    }
    const uint32_t r1 = (mv - 12) / 6, p1 = ((mv - 12) / 2) % 3, p2 = (mv - 12) % 2;
    return {{TD_ROT_BFLY, r1, p1 | (p2 << 2)}, {TD_BFLY_SAME, r1, p1 | (p2 << 2)}, {TD_BFLY_21, r1, p1},
            {TD_BFLY_22, r1, p1}, {TD_BFLY_23_LOZ, r1, p1}, {TD_BFLY_FROM_LOZ, 1, 7u & ~(1u << r1)},
            {TD_TRI_OTHER, 0, 0}};
}

uint32_t mix(uint64_t a, uint64_t b, uint64_t c) {  // splitmix64-style hash of three counters
    uint64_t x = a * 0x9E3779B97F4A7C15ull ^ (b + 0x632BE59BD9B4E019ull) * 0xBF58476D1CE4E5B9ull ^
                 c * 0x94D049BB133111EBull;
    x ^= x >> 31;
    x *= 0xD6E8FEB86659FD93ull;
    x ^= x >> 32;
    return (uint32_t)x;
}

void plane_op(const tdp::View& v, const Phase& p, int m, uint32_t draw) {
    switch (p.op) {
#define RT_CASE(OP)                                        \
    case OP:                                               \
        tdp::word_op<OP>(v, p.a, p.b, m, m, draw);         \
        break;
        RT_CASE(TD_ROT_LOZ)
        RT_CASE(TD_LOZ_FLIPPED)
        RT_CASE(TD_LOZ_OTHER)
        RT_CASE(TD_UP_FROM_LOZ)
        RT_CASE(TD_TRI_OTHER)
        RT_CASE(TD_ROT_TRI)
        RT_CASE(TD_TRI_FLIPPED)
        RT_CASE(TD_LOZ_FROM_TRI)
        RT_CASE(TD_BFLY_FROM_LOZ)
        RT_CASE(TD_ROT_BFLY)
        RT_CASE(TD_BFLY_SAME)
        RT_CASE(TD_BFLY_21)
        RT_CASE(TD_BFLY_22)
        RT_CASE(TD_BFLY_23_LOZ)
#undef RT_CASE
        default: break;
    }
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 4) {
        fprintf(stderr, "usage: tdplane_check ARRAYS_FILE M STEPS | tdplane_check random M ROUNDS\n");
        return 2;
    }
    const int m = atoi(argv[2]), steps = atoi(argv[3]);
    const size_t mm = (size_t)m * m;
    std::vector<int32_t> A(8 * mm), B;
    const bool random = std::string(argv[1]) == "random";
    if (!random) {
        FILE* f = fopen(argv[1], "rb");
        if (!f || fread(A.data(), sizeof(int32_t), A.size(), f) != A.size()) {
            fprintf(stderr, "cannot read %s\n", argv[1]);
            return 2;
        }
        fclose(f);
    }
    // planes: rows -1 .. m (zero halo rows), each row a zero word then wb words then a zero word
    const int wb = (m + 31) / 32, rs = wb + 2, ps = (m + 2) * rs;
    std::vector<uint32_t> P((size_t)tdp::kPlanes * ps);
    auto bit_at = [&](int plane, int i, int j) -> uint32_t& { return P[(size_t)plane * ps + (size_t)(i + 1) * rs + 1 + j / 32]; };
    long checked = 0, changed = 0;
    const int moves = random ? 30 * steps : steps;
    for (int s = 0; s < moves; ++s) {
        const std::vector<Phase> ph = phases_of(s % 30);
        for (size_t q = 0; q < ph.size(); ++q) {
            const Phase& p = ph[q];
            if (random)  // a fresh random state of each array's width before every phase
                for (int arr = 0; arr < 8; ++arr)
                    for (size_t e = 0; e < mm; ++e)
                        A[arr * mm + e] = (int32_t)(mix(0x5eedull + s, q + 97, arr * mm + e) & ((1u << tdp::bits_of(arr)) - 1));
            std::vector<uint32_t> K(mm);
            for (size_t e = 0; e < mm; ++e) K[e] = mix((uint64_t)s, q, e) >> 9;
            // the integer rule, in place (a phase reads no site it writes)
            B = A;
            TriDimerRule::Ctx x;
            x.base = B.data();
            x.plane = (int)mm;
            x.w = m;
            x.m = m;
            x.row0 = 0;
            x.op = p.op;
            x.a = p.a;
            x.b = p.b;
            for (int i = 0; i < m; ++i)
                for (int j = 0; j < m; ++j) TriDimerRule::site_on(x, i, j, K[(size_t)i * m + j]);
            // the bit-plane ops on the old state
            std::fill(P.begin(), P.end(), 0u);
            for (int arr = 0; arr < 8; ++arr)
                for (int k = 0; k < tdp::bits_of(arr); ++k)
                    for (int i = 0; i < m; ++i)
                        for (int j = 0; j < m; ++j)
                            if ((A[arr * mm + (size_t)i * m + j] >> k) & 1)
                                bit_at(tdp::plane_of(arr) + k, i, j) |= 1u << (j % 32);
            for (int i = 0; i < m; ++i)
                for (int c = 0; c < wb; ++c) {
                    uint32_t draw = 0u;
                    for (int l = 0; l < 32; ++l) {
                        const int j = 32 * c + l;
                        if (j < m && K[(size_t)i * m + j] < (1u << 22)) draw |= 1u << l;
                    }
                    const tdp::View v{P.data() + 1, ps, rs, -1, i, c};
                    plane_op(v, p, m, draw);
                }
            for (int arr = 0; arr < 8; ++arr)
                for (int i = 0; i < m; ++i)
                    for (int j = 0; j < m; ++j) {
                        int32_t got = 0;
                        for (int k = 0; k < tdp::bits_of(arr); ++k)
                            if ((bit_at(tdp::plane_of(arr) + k, i, j) >> (j % 32)) & 1u) got |= 1 << k;
                        const size_t at = arr * mm + (size_t)i * m + j;
                        const int32_t want = random ? B[at] & ((1 << tdp::bits_of(arr)) - 1) : B[at];
                        ++checked;
                        changed += B[at] != A[at];
                        if (got != want) {
                            printf("MISMATCH move %d phase %zu (op %u a %u b %u): array %d site (%d, %d): old %d, rule %d, "
                                   "planes %d\n",
                                   s, q, p.op, p.a, p.b, arr, i, j, A[at], B[at], got);
                            return 1;
                        }
                    }
            A.swap(B);
        }
    }
    printf("ok %d moves, %ld values checked, %ld changed\n", moves, checked, changed);
    return 0;
}
