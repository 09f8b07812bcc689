// MRG32k3a (L'Ecuyer 1999; RngStreams, L'Ecuyer, Simard, Chen & Kelton 2002)
// restated with exact 64-bit integer arithmetic. The uniform draw reproduces
// the reference's RngStream::RandU01 with incPrec = true bit for bit
// (CaSim/rngstream.cpp:242-283, 485-491): two recurrence steps per draw,
// u = U01() + U01() * 2^-24, wrapped into [0, 1).
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define CB_HD __host__ __device__ __forceinline__
#else
#define CB_HD inline
#endif

namespace cbrng {

constexpr uint64_t M1 = 4294967087ULL;
constexpr uint64_t M2 = 4294944443ULL;
constexpr uint64_t A12 = 1403580ULL;
constexpr uint64_t A13N = 810728ULL;
constexpr uint64_t A21 = 527612ULL;
constexpr uint64_t A23N = 1370589ULL;

struct State {
    uint32_t s[6];
};

// One recurrence step of both components; returns the combined U(0,1) value.
// Each product is below 2^53 and is reduced on its own, so no intermediate
// exceeds 2^64.
CB_HD double u01(State& g) {
    uint64_t p1 = ((A12 * g.s[1]) % M1 + M1 - (A13N * g.s[0]) % M1) % M1;
    g.s[0] = g.s[1];
    g.s[1] = g.s[2];
    g.s[2] = (uint32_t)p1;
    uint64_t p2 = ((A21 * g.s[5]) % M2 + M2 - (A23N * g.s[3]) % M2) % M2;
    g.s[3] = g.s[4];
    g.s[4] = g.s[5];
    g.s[5] = (uint32_t)p2;
    const double norm = 1.0 / (4294967087.0 + 1.0);
    double d1 = (double)p1, d2 = (double)p2;
#ifdef __CUDA_ARCH__
    return (p1 > p2) ? __dmul_rn(d1 - d2, norm) : __dmul_rn(__dadd_rn(d1 - d2, 4294967087.0), norm);
#else
    return (p1 > p2) ? (d1 - d2) * norm : (d1 - d2 + 4294967087.0) * norm;
#endif
}

// RandU01 with increased precision: no FMA contraction of u + v * 2^-24.
CB_HD double u01d(State& g) {
    const double fact = 5.9604644775390625e-8;  // 2^-24
    double u = u01(g);
    double v = u01(g);
#ifdef __CUDA_ARCH__
    u = __dadd_rn(u, __dmul_rn(v, fact));
#else
    u = u + v * fact;
#endif
    return (u < 1.0) ? u : (u - 1.0);
}

#ifdef __CUDACC__
// The same recurrence with the modular products reduced by folding
// (m = 2^32 - c: x = hi * 2^32 + lo == hi * c + lo), two folds and one
// conditional subtraction instead of 64-bit remainders; bit-identical draws.
template <uint64_t M>
__device__ __forceinline__ uint64_t fold_mod(uint64_t x) {
    constexpr uint64_t c = (1ULL << 32) - M;
    uint64_t t = (x >> 32) * c + (x & 0xffffffffULL);
    t = (t >> 32) * c + (t & 0xffffffffULL);
    return t >= M ? t - M : t;
}

__device__ __forceinline__ double u01_fold(State& g) {
    uint64_t a = fold_mod<M1>(A12 * g.s[1]);
    uint64_t b = fold_mod<M1>(A13N * g.s[0]);
    const uint64_t p1 = a >= b ? a - b : a + M1 - b;
    g.s[0] = g.s[1];
    g.s[1] = g.s[2];
    g.s[2] = (uint32_t)p1;
    a = fold_mod<M2>(A21 * g.s[5]);
    b = fold_mod<M2>(A23N * g.s[3]);
    const uint64_t p2 = a >= b ? a - b : a + M2 - b;
    g.s[3] = g.s[4];
    g.s[4] = g.s[5];
    g.s[5] = (uint32_t)p2;
    const double norm = 1.0 / (4294967087.0 + 1.0);
    const double d1 = (double)p1, d2 = (double)p2;
    return (p1 > p2) ? __dmul_rn(d1 - d2, norm) : __dmul_rn(__dadd_rn(d1 - d2, 4294967087.0), norm);
}

// u01d with the folding recurrence (CaSim/rngstream.cpp:271-283, incPrec)
__device__ __forceinline__ double u01d_fold(State& g) {
    double u = u01_fold(g);
    const double v = u01_fold(g);
    u = __dadd_rn(u, __dmul_rn(v, 5.9604644775390625e-8));
    return (u < 1.0) ? u : (u - 1.0);
}

// v = A v (mod M) for a 3x3 jump matrix A (row-major, entries < M) of one component
template <uint64_t M>
__device__ __forceinline__ void mat_apply(const unsigned long long* A, unsigned int* v) {
    unsigned long long r[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        unsigned long long acc = 0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            acc += fold_mod<M>(A[3 * i + k] * (unsigned long long)v[k]);
            if (acc >= M) acc -= M;
        }
        r[i] = acc;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) v[i] = (unsigned int)r[i];
}

// advance both components by the jump stored at J (18 entries: A1 then A2)
__device__ __forceinline__ void jump_by(const unsigned long long* J, State& g) {
    mat_apply<M1>(J, g.s);
    mat_apply<M2>(J + 9, g.s + 3);
}
#endif

// ---- host-side jump-ahead (3x3 matrix powers of the two recurrences) ----
struct Mat3 {
    uint64_t a[3][3];
};

inline uint64_t mulmod(uint64_t a, uint64_t b, uint64_t m) { return (uint64_t)(((unsigned __int128)a * b) % m); }

inline Mat3 matmul(const Mat3& x, const Mat3& y, uint64_t m) {
    Mat3 r{};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            uint64_t acc = 0;
            for (int k = 0; k < 3; ++k) acc = (acc + mulmod(x.a[i][k], y.a[k][j], m)) % m;
            r.a[i][j] = acc;
        }
    return r;
}

inline void matvec(const Mat3& x, uint64_t* v, uint64_t m) {
    uint64_t r[3];
    for (int i = 0; i < 3; ++i) {
        uint64_t acc = 0;
        for (int k = 0; k < 3; ++k) acc = (acc + mulmod(x.a[i][k], v[k], m)) % m;
        r[i] = acc;
    }
    for (int i = 0; i < 3; ++i) v[i] = r[i];
}

inline Mat3 step_matrix1() { return Mat3{{{0, 1, 0}, {0, 0, 1}, {M1 - A13N, A12, 0}}}; }
inline Mat3 step_matrix2() { return Mat3{{{0, 1, 0}, {0, 0, 1}, {M2 - A23N, 0, A21}}}; }

// Advance `st` by 2^e recurrence steps, `times` times.
inline void jump_pow2(State& st, int e, uint64_t times) {
    Mat3 a1 = step_matrix1(), a2 = step_matrix2();
    for (int i = 0; i < e; ++i) {
        a1 = matmul(a1, a1, M1);
        a2 = matmul(a2, a2, M2);
    }
    uint64_t v1[3] = {st.s[0], st.s[1], st.s[2]}, v2[3] = {st.s[3], st.s[4], st.s[5]};
    for (uint64_t k = 0; k < times; ++k) {
        matvec(a1, v1, M1);
        matvec(a2, v2, M2);
    }
    for (int i = 0; i < 3; ++i) {
        st.s[i] = (uint32_t)v1[i];
        st.s[i + 3] = (uint32_t)v2[i];
    }
}

// RngStreams seed validity (CaSim/rngstream.cpp:200-234).
inline bool seed_ok(const uint64_t s[6]) {
    for (int i = 0; i < 3; ++i)
        if (s[i] >= M1) return false;
    for (int i = 3; i < 6; ++i)
        if (s[i] >= M2) return false;
    if (s[0] == 0 && s[1] == 0 && s[2] == 0) return false;
    if (s[3] == 0 && s[4] == 0 && s[5] == 0) return false;
    return true;
}

}  // namespace cbrng
