// BN254 Fr / Fq / Fq2 arithmetic for sm_100a.
//
// Eight 32-bit little-endian limbs, Montgomery form with R = 2^256: the same
// bits as arkworks' in-memory Fp and snarkrs' PackedFr / PackedFq
// (crates/gpu-layout/src/lib.rs:30-46, 75-113).  Every value leaving a
// function is fully reduced into [0, p), so device results compare bit for
// bit with the CPU prover.
//
// The Montgomery product is CIOS (Koc, Acar and Kaliski, "Analyzing and
// comparing Montgomery multiplication algorithms", 1996) in two forms with
// identical results:
//   * mul_cc: PTX multiply-add carry chains -- per limb of b, one
//     mad.lo.cc/madc.lo.cc chain and one mad.hi.cc/madc.hi.cc chain for
//     a*b[i], then the same pair for m*p, each chain in one asm statement.
//     Used by the NTT butterflies.
//   * mul: the same CIOS on 32x32->64-bit multiply-adds with the carries in
//     64-bit sums, which the compiler lowers to wide IMADs plus 3-input adds
//     on the ALU pipe.  On sm_100a it measured 843 cycles for one warp's
//     dependent product against 1381 for mul_cc, 45.8 against 43.7 G
//     products/s at full occupancy, and 5-38% faster MSM kernels, so every
//     point formula uses it.
// BN254's moduli are below 2^254, so the running sum stays below 2^287 and
// fits nine limbs; the carry out of the ninth is provably zero.
#pragma once
#include <cstdint>

namespace g16d {

// Limb tables as constexpr functions: every use sits in a fully unrolled loop
// or an "n" asm operand, so each call folds to an immediate.
struct FrParams {
    __host__ __device__ static constexpr uint32_t P(int i) {
        constexpr uint32_t v[8] = {0xf0000001u, 0x43e1f593u, 0x79b97091u, 0x2833e848u,
                                   0x8181585du, 0xb85045b6u, 0xe131a029u, 0x30644e72u};
        return v[i];
    }
    static constexpr uint32_t N0 = 0xefffffffu;
    // R mod r, the Montgomery form of one
    __host__ __device__ static constexpr uint32_t ONE(int i) {
        constexpr uint32_t v[8] = {0x4ffffffbu, 0xac96341cu, 0x9f60cd29u, 0x36fc7695u,
                                   0x7879462eu, 0x666ea36fu, 0x9a07df2fu, 0x0e0a77c1u};
        return v[i];
    }
};

struct FqParams {
    __host__ __device__ static constexpr uint32_t P(int i) {
        constexpr uint32_t v[8] = {0xd87cfd47u, 0x3c208c16u, 0x6871ca8du, 0x97816a91u,
                                   0x8181585du, 0xb85045b6u, 0xe131a029u, 0x30644e72u};
        return v[i];
    }
    static constexpr uint32_t N0 = 0xe4866389u;
    __host__ __device__ static constexpr uint32_t ONE(int i) {
        constexpr uint32_t v[8] = {0xc58f0d9du, 0xd35d438du, 0xf5c70b3du, 0x0a78eb28u,
                                   0x7879462cu, 0x666ea36fu, 0x9a07df2fu, 0x0e0a77c1u};
        return v[i];
    }
    // q^2 as 16 limbs (the Fq2 product's offset that keeps a0 b0 - a1 b1 positive)
    __host__ __device__ static constexpr uint32_t P2W(int i) {
        constexpr uint32_t v[16] = {0x275d69b1u, 0x3b5458a2u, 0x09eac101u, 0xa602072du, 0x6d96cadcu, 0x4a50189cu,
                                    0x7a1242c8u, 0x04689e95u, 0x34c6b38du, 0x26edfa5cu, 0x16375606u, 0xb00b8551u,
                                    0x0348d21cu, 0x599a6f7cu, 0x763cbf9cu, 0x0925c4b8u};
        return v[i];
    }
};

template <class Params>
struct __align__(16) Fp {
    uint32_t v[8];

    __device__ __forceinline__ static Fp zero() {
        Fp r;
#pragma unroll
        for (int i = 0; i < 8; i++) r.v[i] = 0;
        return r;
    }
    __device__ __forceinline__ static Fp one() {
        Fp r;
#pragma unroll
        for (int i = 0; i < 8; i++) r.v[i] = Params::ONE(i);
        return r;
    }
    __device__ __forceinline__ bool is_zero() const {
        uint32_t acc = v[0];
#pragma unroll
        for (int i = 1; i < 8; i++) acc |= v[i];
        return acc == 0;
    }
    __device__ __forceinline__ bool eq(const Fp& o) const {
        uint32_t acc = 0;
#pragma unroll
        for (int i = 0; i < 8; i++) acc |= v[i] ^ o.v[i];
        return acc == 0;
    }
    __device__ __forceinline__ bool is_one() const { return eq(one()); }
};

// r = a - p if a >= p (a < 2p), in registers
template <class Params>
__device__ __forceinline__ void reduce_once(uint32_t* a) {
    uint32_t d[8], borrow;
    asm("sub.cc.u32  %0, %9, %17;\n\t"
        "subc.cc.u32 %1, %10, %18;\n\t"
        "subc.cc.u32 %2, %11, %19;\n\t"
        "subc.cc.u32 %3, %12, %20;\n\t"
        "subc.cc.u32 %4, %13, %21;\n\t"
        "subc.cc.u32 %5, %14, %22;\n\t"
        "subc.cc.u32 %6, %15, %23;\n\t"
        "subc.cc.u32 %7, %16, %24;\n\t"
        "subc.u32    %8, 0, 0;"
        : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
          "=r"(borrow)
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]),
          "n"(Params::P(0)), "n"(Params::P(1)), "n"(Params::P(2)), "n"(Params::P(3)), "n"(Params::P(4)),
          "n"(Params::P(5)), "n"(Params::P(6)), "n"(Params::P(7)));
    // borrow == 0xffffffff when a < p: keep a
#pragma unroll
    for (int i = 0; i < 8; i++) a[i] = borrow ? a[i] : d[i];
}

template <class Params>
__device__ __forceinline__ Fp<Params> add(const Fp<Params>& a, const Fp<Params>& b) {
    Fp<Params> r;
    asm("add.cc.u32  %0, %8, %16;\n\t"
        "addc.cc.u32 %1, %9, %17;\n\t"
        "addc.cc.u32 %2, %10, %18;\n\t"
        "addc.cc.u32 %3, %11, %19;\n\t"
        "addc.cc.u32 %4, %12, %20;\n\t"
        "addc.cc.u32 %5, %13, %21;\n\t"
        "addc.cc.u32 %6, %14, %22;\n\t"
        "addc.u32    %7, %15, %23;"
        : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]), "=r"(r.v[6]),
          "=r"(r.v[7])
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]), "r"(a.v[7]),
          "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]), "r"(b.v[6]), "r"(b.v[7]));
    reduce_once<Params>(r.v);
    return r;
}

template <class Params>
__device__ __forceinline__ Fp<Params> sub(const Fp<Params>& a, const Fp<Params>& b) {
    Fp<Params> r;
    uint32_t borrow;
    asm("sub.cc.u32  %0, %9, %17;\n\t"
        "subc.cc.u32 %1, %10, %18;\n\t"
        "subc.cc.u32 %2, %11, %19;\n\t"
        "subc.cc.u32 %3, %12, %20;\n\t"
        "subc.cc.u32 %4, %13, %21;\n\t"
        "subc.cc.u32 %5, %14, %22;\n\t"
        "subc.cc.u32 %6, %15, %23;\n\t"
        "subc.cc.u32 %7, %16, %24;\n\t"
        "subc.u32    %8, 0, 0;"
        : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]), "=r"(r.v[6]),
          "=r"(r.v[7]), "=r"(borrow)
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]), "r"(a.v[7]),
          "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]), "r"(b.v[6]), "r"(b.v[7]));
    // add p back when the subtraction borrowed (p & mask)
    uint32_t m = borrow;
    asm("add.cc.u32  %0, %0, %8;\n\t"
        "addc.cc.u32 %1, %1, %9;\n\t"
        "addc.cc.u32 %2, %2, %10;\n\t"
        "addc.cc.u32 %3, %3, %11;\n\t"
        "addc.cc.u32 %4, %4, %12;\n\t"
        "addc.cc.u32 %5, %5, %13;\n\t"
        "addc.cc.u32 %6, %6, %14;\n\t"
        "addc.u32    %7, %7, %15;"
        : "+r"(r.v[0]), "+r"(r.v[1]), "+r"(r.v[2]), "+r"(r.v[3]), "+r"(r.v[4]), "+r"(r.v[5]), "+r"(r.v[6]),
          "+r"(r.v[7])
        : "r"(Params::P(0) & m), "r"(Params::P(1) & m), "r"(Params::P(2) & m), "r"(Params::P(3) & m),
          "r"(Params::P(4) & m), "r"(Params::P(5) & m), "r"(Params::P(6) & m), "r"(Params::P(7) & m));
    return r;
}

template <class Params>
__device__ __forceinline__ Fp<Params> neg(const Fp<Params>& a) {
    return a.is_zero() ? a : sub(Fp<Params>::zero(), a);
}

template <class Params>
__device__ __forceinline__ Fp<Params> dbl(const Fp<Params>& a) {
    return add(a, a);
}

// t[0..8] += a[0..7] * b  (lo halves into t0..t7 with carry into t8, then hi halves into t1..t8)
#define G16_MAD_ROW(T, A, B)                                                                         \
    asm("mad.lo.cc.u32  %0, %9, %17, %0;\n\t"                                                        \
        "madc.lo.cc.u32 %1, %10, %17, %1;\n\t"                                                       \
        "madc.lo.cc.u32 %2, %11, %17, %2;\n\t"                                                       \
        "madc.lo.cc.u32 %3, %12, %17, %3;\n\t"                                                       \
        "madc.lo.cc.u32 %4, %13, %17, %4;\n\t"                                                       \
        "madc.lo.cc.u32 %5, %14, %17, %5;\n\t"                                                       \
        "madc.lo.cc.u32 %6, %15, %17, %6;\n\t"                                                       \
        "madc.lo.cc.u32 %7, %16, %17, %7;\n\t"                                                       \
        "addc.u32       %8, %8, 0;\n\t"                                                              \
        "mad.hi.cc.u32  %1, %9, %17, %1;\n\t"                                                        \
        "madc.hi.cc.u32 %2, %10, %17, %2;\n\t"                                                       \
        "madc.hi.cc.u32 %3, %11, %17, %3;\n\t"                                                       \
        "madc.hi.cc.u32 %4, %12, %17, %4;\n\t"                                                       \
        "madc.hi.cc.u32 %5, %13, %17, %5;\n\t"                                                       \
        "madc.hi.cc.u32 %6, %14, %17, %6;\n\t"                                                       \
        "madc.hi.cc.u32 %7, %15, %17, %7;\n\t"                                                       \
        "madc.hi.u32    %8, %16, %17, %8;"                                                           \
        : "+r"(T[0]), "+r"(T[1]), "+r"(T[2]), "+r"(T[3]), "+r"(T[4]), "+r"(T[5]), "+r"(T[6]),        \
          "+r"(T[7]), "+r"(T[8])                                                                     \
        : "r"(A[0]), "r"(A[1]), "r"(A[2]), "r"(A[3]), "r"(A[4]), "r"(A[5]), "r"(A[6]), "r"(A[7]),    \
          "r"(B))

// t[0..8] += m * P, then shift down one limb
#define G16_REDUCE_ROW(T, M, PP)                                                                     \
    asm("mad.lo.cc.u32  %0, %9, %10, %0;\n\t"                                                        \
        "madc.lo.cc.u32 %1, %9, %11, %1;\n\t"                                                        \
        "madc.lo.cc.u32 %2, %9, %12, %2;\n\t"                                                        \
        "madc.lo.cc.u32 %3, %9, %13, %3;\n\t"                                                        \
        "madc.lo.cc.u32 %4, %9, %14, %4;\n\t"                                                        \
        "madc.lo.cc.u32 %5, %9, %15, %5;\n\t"                                                        \
        "madc.lo.cc.u32 %6, %9, %16, %6;\n\t"                                                        \
        "madc.lo.cc.u32 %7, %9, %17, %7;\n\t"                                                        \
        "addc.u32       %8, %8, 0;\n\t"                                                              \
        "mad.hi.cc.u32  %1, %9, %10, %1;\n\t"                                                        \
        "madc.hi.cc.u32 %2, %9, %11, %2;\n\t"                                                        \
        "madc.hi.cc.u32 %3, %9, %12, %3;\n\t"                                                        \
        "madc.hi.cc.u32 %4, %9, %13, %4;\n\t"                                                        \
        "madc.hi.cc.u32 %5, %9, %14, %5;\n\t"                                                        \
        "madc.hi.cc.u32 %6, %9, %15, %6;\n\t"                                                        \
        "madc.hi.cc.u32 %7, %9, %16, %7;\n\t"                                                        \
        "madc.hi.u32    %8, %9, %17, %8;"                                                            \
        : "+r"(T[0]), "+r"(T[1]), "+r"(T[2]), "+r"(T[3]), "+r"(T[4]), "+r"(T[5]), "+r"(T[6]),        \
          "+r"(T[7]), "+r"(T[8])                                                                     \
        : "r"(M), "n"(PP::P(0)), "n"(PP::P(1)), "n"(PP::P(2)), "n"(PP::P(3)), "n"(PP::P(4)),         \
          "n"(PP::P(5)), "n"(PP::P(6)), "n"(PP::P(7)))

template <class Params>
__device__ __forceinline__ Fp<Params> mul_cc(const Fp<Params>& a, const Fp<Params>& b) {
    uint32_t t[9];
#pragma unroll
    for (int i = 0; i < 9; i++) t[i] = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        G16_MAD_ROW(t, a.v, b.v[i]);
        uint32_t m = t[0] * Params::N0;
        G16_REDUCE_ROW(t, m, Params);
        // t0 is now zero: shift down
#pragma unroll
        for (int j = 0; j < 8; j++) t[j] = t[j + 1];
        t[8] = 0;
    }
    reduce_once<Params>(t);
    Fp<Params> r;
#pragma unroll
    for (int i = 0; i < 8; i++) r.v[i] = t[i];
    return r;
}

// CIOS with 64-bit sums: t[j] + a[j] b[i] + carry < 2^64 always holds
template <class Params>
__device__ __forceinline__ Fp<Params> mul(const Fp<Params>& a, const Fp<Params>& b) {
    uint32_t t[10];
#pragma unroll
    for (int i = 0; i < 10; i++) t[i] = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        uint64_t c = 0;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            uint64_t p = (uint64_t)a.v[j] * b.v[i] + t[j] + c;
            t[j] = (uint32_t)p;
            c = p >> 32;
        }
        uint64_t s = (uint64_t)t[8] + c;
        t[8] = (uint32_t)s;
        t[9] = (uint32_t)(s >> 32);
        // m = t0 * (-p^-1) mod 2^32 makes t + m p divisible by 2^32
        uint32_t m = t[0] * Params::N0;
        c = ((uint64_t)m * Params::P(0) + t[0]) >> 32;
#pragma unroll
        for (int j = 1; j < 8; j++) {
            uint64_t p = (uint64_t)m * Params::P(j) + t[j] + c;
            t[j - 1] = (uint32_t)p;
            c = p >> 32;
        }
        s = (uint64_t)t[8] + c;
        t[7] = (uint32_t)s;
        t[8] = t[9] + (uint32_t)(s >> 32);
    }
    reduce_once<Params>(t);
    Fp<Params> r;
#pragma unroll
    for (int i = 0; i < 8; i++) r.v[i] = t[i];
    return r;
}

// Montgomery reduction of a 16-limb t < p R: t R^-1 mod p, left in [0, 2p)
// in r[0..7] (t is clobbered).  Row i adds m p 2^(32 i), m = t[i] (-p^-1) mod
// 2^32, which zeroes limb i; the carry out of limb i + 8 rides into the next
// row.  (t + M p) / R < 2p < 2^255, so no carry is left at the end.
template <class Params>
__host__ __device__ __forceinline__ void redc_wide(uint32_t* t, uint32_t* r) {
    uint32_t extra = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        uint32_t m = t[i] * Params::N0;
        uint64_t c = ((uint64_t)m * Params::P(0) + t[i]) >> 32;
#pragma unroll
        for (int j = 1; j < 8; j++) {
            uint64_t p = (uint64_t)m * Params::P(j) + t[i + j] + c;
            t[i + j] = (uint32_t)p;
            c = p >> 32;
        }
        uint64_t s = (uint64_t)t[i + 8] + c + extra;
        t[i + 8] = (uint32_t)s;
        extra = (uint32_t)(s >> 32);
    }
#pragma unroll
    for (int k = 0; k < 8; k++) r[k] = t[k + 8];
}

// a b as a 16-limb integer (schoolbook rows with 64-bit sums; row i writes
// limb i + 8 fresh, since the rows before it reach limb i + 7 at most)
__host__ __device__ __forceinline__ void mul_wide(const uint32_t* a, const uint32_t* b, uint32_t* t) {
#pragma unroll
    for (int k = 0; k < 16; k++) t[k] = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        uint64_t c = 0;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            uint64_t p = (uint64_t)a[j] * b[i] + t[i + j] + c;
            t[i + j] = (uint32_t)p;
            c = p >> 32;
        }
        t[i + 8] = (uint32_t)c;
    }
}

// a^2 R^-1 mod p, left in [0, 2p) in r[0..7] (separated operand scanning):
// the 28 cross products a_i a_j (i < j) once, doubled by a one-bit shift, plus
// the 8 squares a_i^2, then a Montgomery reduction of the 16-limb square.  36
// limb products and 64 for the reduction against CIOS's 128: the same REDC
// value (a^2 + M p) / R, M being the unique multiple in [0, R), so the result
// is identical to mul(a, a).  Host-callable for the unit check of the limbs.
template <class Params>
__host__ __device__ __forceinline__ void sqr_redc(const uint32_t* a, uint32_t* r) {
    uint32_t t[16];
#pragma unroll
    for (int k = 0; k < 16; k++) t[k] = 0;
    // cross products: row i adds a_i a_j (j > i) at limb i + j; t[i + 8] is untouched before row i
#pragma unroll
    for (int i = 0; i < 7; i++) {
        uint64_t c = 0;
#pragma unroll
        for (int j = i + 1; j < 8; j++) {
            uint64_t p = (uint64_t)a[i] * a[j] + t[i + j] + c;
            t[i + j] = (uint32_t)p;
            c = p >> 32;
        }
        t[i + 8] = (uint32_t)c;
    }
    // double (the cross sum is below 2^511, so the shift loses nothing)
    t[15] = t[14] >> 31;
#pragma unroll
    for (int k = 14; k >= 1; k--) t[k] = (t[k] << 1) | (t[k - 1] >> 31);
    // t[0] is zero: no cross product lands on limb 0
    // add the squares a_i^2 at limbs 2i, 2i + 1
    {
        uint64_t c = 0;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            uint64_t q = (uint64_t)a[i] * a[i];
            uint64_t s0 = (uint64_t)t[2 * i] + (uint32_t)q + c;
            t[2 * i] = (uint32_t)s0;
            uint64_t s1 = (uint64_t)t[2 * i + 1] + (q >> 32) + (s0 >> 32);
            t[2 * i + 1] = (uint32_t)s1;
            c = s1 >> 32;
        }
    }
    redc_wide<Params>(t, r);
}

template <class Params>
__device__ __forceinline__ Fp<Params> sqr(const Fp<Params>& a) {
    Fp<Params> r;
    sqr_redc<Params>(a.v, r.v);
    reduce_once<Params>(r.v);
    return r;
}

// Montgomery -> standard form: a * 1 * R^-1
template <class Params>
__device__ __forceinline__ Fp<Params> from_mont(const Fp<Params>& a) {
    Fp<Params> one_raw = Fp<Params>::zero();
    one_raw.v[0] = 1;
    return mul(a, one_raw);
}

typedef Fp<FrParams> Fr;
typedef Fp<FqParams> Fq;

// ---- Fq2 = Fq[u]/(u^2 + 1) ----
struct __align__(16) Fq2 {
    Fq c0, c1;
    __device__ __forceinline__ static Fq2 zero() { return {Fq::zero(), Fq::zero()}; }
    __device__ __forceinline__ static Fq2 one() { return {Fq::one(), Fq::zero()}; }
    __device__ __forceinline__ bool is_zero() const { return c0.is_zero() && c1.is_zero(); }
};

__device__ __forceinline__ Fq2 add(const Fq2& a, const Fq2& b) { return {add(a.c0, b.c0), add(a.c1, b.c1)}; }
__device__ __forceinline__ Fq2 sub(const Fq2& a, const Fq2& b) { return {sub(a.c0, b.c0), sub(a.c1, b.c1)}; }
__device__ __forceinline__ Fq2 neg(const Fq2& a) { return {neg(a.c0), neg(a.c1)}; }
__device__ __forceinline__ Fq2 dbl(const Fq2& a) { return {dbl(a.c0), dbl(a.c1)}; }
// (a b - c d) R^-1 mod p, left in [0, 2p), with one Montgomery reduction
// instead of two: the 512-bit a b + p^2 - c d is positive and below 2 p^2 < p R
// for inputs below p, and its reduction equals (a b R^-1 - c d R^-1) mod p.
// c d is subtracted row by row; the borrow out of limb i + 8 rides into the
// next row, as the carry does in redc_wide (the running value never drops
// below a b + p^2 - c d > 0).  Params must carry p^2 (P2W).  Host-callable.
template <class Params>
__host__ __device__ __forceinline__ void mul_sub_redc(const uint32_t* a, const uint32_t* b, const uint32_t* c,
                                                      const uint32_t* d, uint32_t* r) {
    uint32_t t[16];
    mul_wide(a, b, t);
    {
        uint64_t k = 0;
#pragma unroll
        for (int i = 0; i < 16; i++) {
            k += (uint64_t)t[i] + Params::P2W(i);
            t[i] = (uint32_t)k;
            k >>= 32;
        }
    }
    int64_t pend = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        uint64_t cy = 0;
        int64_t br = 0;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            uint64_t pr = (uint64_t)c[j] * d[i] + cy;
            cy = pr >> 32;
            int64_t x = (int64_t)t[i + j] - (int64_t)(uint32_t)pr + br;
            t[i + j] = (uint32_t)x;
            br = x >> 32;
        }
        int64_t x = (int64_t)t[i + 8] - (int64_t)cy + br + pend;
        t[i + 8] = (uint32_t)x;
        pend = x >> 32;
    }
    redc_wide<Params>(t, r);
}

// a b - c d in Fq with one reduction (mul_sub_redc)
__device__ __forceinline__ Fq mul_sub(const Fq& a, const Fq& b, const Fq& c, const Fq& d) {
    Fq r;
    mul_sub_redc<FqParams>(a.v, b.v, c.v, d.v, r.v);
    reduce_once<FqParams>(r.v);
    return r;
}

// (a0 + a1 u)(b0 + b1 u) with two Montgomery reductions instead of three
// (Karatsuba with the reduction deferred, as in Aranha et al., "Faster explicit
// formulas for computing pairings over ordinary curves", 2011): the three
// 512-bit products t0 = a0 b0, t1 = a1 b1, m = (a0 + a1)(b0 + b1) with the
// sums taken as integers (below 2q), then
//   c1 = m - t0 - t1 = a0 b1 + a1 b0          (exact, below 2 q^2)
//   c0 = t0 + q^2 - t1 = a0 b0 - a1 b1 mod q  (positive, below 2 q^2),
// and one reduction each (inputs below q R give results below 2q).  The
// coordinates equal those of three reduced products once brought below q.
// Inputs below q.  Host-callable for the unit check of the limbs.
__host__ __device__ __forceinline__ void fq2_mul_redc(const uint32_t* a0, const uint32_t* a1, const uint32_t* b0,
                                                      const uint32_t* b1, uint32_t* r0, uint32_t* r1) {
    uint32_t t0[16], t1[16], m[16], sa[8], sb[8];
    {
        uint64_t ca = 0, cb = 0;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            ca += (uint64_t)a0[i] + a1[i];
            sa[i] = (uint32_t)ca;
            ca >>= 32;
            cb += (uint64_t)b0[i] + b1[i];
            sb[i] = (uint32_t)cb;
            cb >>= 32;
        }
    }
    mul_wide(a0, b0, t0);
    mul_wide(a1, b1, t1);
    mul_wide(sa, sb, m);
    // m -= t0 + t1;  t0 += q^2 - t1
    {
        int64_t bm = 0, b0w = 0;
#pragma unroll
        for (int i = 0; i < 16; i++) {
            int64_t dm = (int64_t)m[i] - t0[i] - t1[i] + bm;
            m[i] = (uint32_t)dm;
            bm = dm >> 32;   // arithmetic shift: 0, -1 or -2
            int64_t d0 = (int64_t)t0[i] + FqParams::P2W(i) - t1[i] + b0w;
            t0[i] = (uint32_t)d0;
            b0w = d0 >> 32;  // -1, 0 or 1
        }
    }
    redc_wide<FqParams>(t0, r0);
    redc_wide<FqParams>(m, r1);
}

__device__ __forceinline__ Fq2 mul(const Fq2& a, const Fq2& b) {
    Fq2 r;
    fq2_mul_redc(a.c0.v, a.c1.v, b.c0.v, b.c1.v, r.c0.v, r.c1.v);
    reduce_once<FqParams>(r.c0.v);
    reduce_once<FqParams>(r.c1.v);
    return r;
}
// a b - c d in Fq2: two products and a difference
__device__ __forceinline__ Fq2 mul_sub(const Fq2& a, const Fq2& b, const Fq2& c, const Fq2& d) {
    return sub(mul(a, b), mul(c, d));
}
// (a0 + a1 u)^2 = (a0 + a1)(a0 - a1) + 2 a0 a1 u
__device__ __forceinline__ Fq2 sqr(const Fq2& a) {
    Fq p = mul(add(a.c0, a.c1), sub(a.c0, a.c1));
    Fq q = mul(a.c0, a.c1);
    return {p, dbl(q)};
}

// ---- product policy: inlined, or one out-of-line copy ----
// Latency-bound kernels (bucket reduction) run long dependent chains of point
// operations; inlining ~14 CIOS bodies per point operation, several operations
// per kernel, overflows the instruction cache.  They call a single
// out-of-line copy instead (operands by value, so they stay in registers).
// The throughput kernels keep every product inlined.
template <class Params>
__device__ __noinline__ Fp<Params> mul_ool(Fp<Params> a, Fp<Params> b) {
    return mul(a, b);
}

template <bool INL, class Params>
__device__ __forceinline__ Fp<Params> fmul(const Fp<Params>& a, const Fp<Params>& b) {
    if constexpr (INL) return mul(a, b);
    else return mul_ool(a, b);
}
template <bool INL, class Params>
__device__ __forceinline__ Fp<Params> fsqr(const Fp<Params>& a) {
    if constexpr (INL) return sqr(a);
    else return mul_ool(a, a);
}

// Out-of-line copies that hold several independent products.  A warp issues
// in order and a CIOS product is one long carry chain, so a lone out-of-line
// product leaves the pipe idle for most of its latency; two or three chains in
// one body are scheduled side by side.  The latency-bound kernels group the
// independent products of each point formula this way.
template <class F>
struct Two {
    F a, b;
};
template <class F>
struct Three {
    F a, b, c;
};

template <class Params>
__device__ __noinline__ Two<Fp<Params>> mul2_ool(Fp<Params> a0, Fp<Params> b0, Fp<Params> a1, Fp<Params> b1) {
    return {mul(a0, b0), mul(a1, b1)};
}
template <class Params>
__device__ __noinline__ Three<Fp<Params>> mul3_ool(Fp<Params> a0, Fp<Params> b0, Fp<Params> a1, Fp<Params> b1,
                                                   Fp<Params> a2, Fp<Params> b2) {
    return {mul(a0, b0), mul(a1, b1), mul(a2, b2)};
}
// an Fq2 product is already three independent Fq products (Karatsuba)
static __device__ __noinline__ Fq2 fq2_mul_ool(Fq2 a, Fq2 b) { return mul(a, b); }
static __device__ __noinline__ Fq2 fq2_sqr_ool(Fq2 a) { return sqr(a); }

template <bool INL>
__device__ __forceinline__ Fq2 fmul(const Fq2& a, const Fq2& b) {
    if constexpr (INL) return mul(a, b);
    else return fq2_mul_ool(a, b);
}
template <bool INL>
__device__ __forceinline__ Fq2 fsqr(const Fq2& a) {
    if constexpr (INL) return sqr(a);
    else return fq2_sqr_ool(a);
}

// r0 = a0 b0, r1 = a1 b1 (and r2 = a2 b2), independent products side by side
template <bool INL, class Params>
__device__ __forceinline__ void fmul2(const Fp<Params>& a0, const Fp<Params>& b0, const Fp<Params>& a1,
                                      const Fp<Params>& b1, Fp<Params>& r0, Fp<Params>& r1) {
    if constexpr (INL) {
        r0 = mul(a0, b0);
        r1 = mul(a1, b1);
    } else {
        Two<Fp<Params>> t = mul2_ool(a0, b0, a1, b1);
        r0 = t.a;
        r1 = t.b;
    }
}
template <bool INL, class Params>
__device__ __forceinline__ void fmul3(const Fp<Params>& a0, const Fp<Params>& b0, const Fp<Params>& a1,
                                      const Fp<Params>& b1, const Fp<Params>& a2, const Fp<Params>& b2,
                                      Fp<Params>& r0, Fp<Params>& r1, Fp<Params>& r2) {
    if constexpr (INL) {
        r0 = mul(a0, b0);
        r1 = mul(a1, b1);
        r2 = mul(a2, b2);
    } else {
        Three<Fp<Params>> t = mul3_ool(a0, b0, a1, b1, a2, b2);
        r0 = t.a;
        r1 = t.b;
        r2 = t.c;
    }
}
template <bool INL>
__device__ __forceinline__ void fmul2(const Fq2& a0, const Fq2& b0, const Fq2& a1, const Fq2& b1, Fq2& r0, Fq2& r1) {
    r0 = fmul<INL>(a0, b0);
    r1 = fmul<INL>(a1, b1);
}
template <bool INL>
__device__ __forceinline__ void fmul3(const Fq2& a0, const Fq2& b0, const Fq2& a1, const Fq2& b1, const Fq2& a2,
                                      const Fq2& b2, Fq2& r0, Fq2& r1, Fq2& r2) {
    r0 = fmul<INL>(a0, b0);
    r1 = fmul<INL>(a1, b1);
    r2 = fmul<INL>(a2, b2);
}

// a^(p-2) by right-to-left square-and-multiply (Fermat); 0 maps to 0.  Used
// off the hot path (table building), so it calls the out-of-line product.
template <class Params>
__device__ Fp<Params> inv(const Fp<Params>& a) {
    Fp<Params> r = Fp<Params>::one(), b = a;
#pragma unroll
    for (int limb = 0; limb < 8; limb++) {
        uint32_t e = Params::P(limb) - (limb == 0 ? 2u : 0u);
        for (int bit = 0; bit < 32; bit++) {
            if (e & 1u) r = mul_ool(r, b);
            b = mul_ool(b, b);
            e >>= 1;
        }
    }
    return r;
}

// 1/(c0 + c1 u) = (c0 - c1 u) / (c0^2 + c1^2)
__device__ __forceinline__ Fq2 inv(const Fq2& a) {
    Fq n = inv(add(mul_ool(a.c0, a.c0), mul_ool(a.c1, a.c1)));
    return {mul_ool(a.c0, n), neg(mul_ool(a.c1, n))};
}

// ---- 128-bit vector loads / stores of 32-byte elements ----
template <class T>
__device__ __forceinline__ T load32(const T* p) {
    static_assert(sizeof(T) == 32, "32-byte element");
    const uint4* q = reinterpret_cast<const uint4*>(p);
    uint4 lo = q[0], hi = q[1];
    T r;
    r.v[0] = lo.x; r.v[1] = lo.y; r.v[2] = lo.z; r.v[3] = lo.w;
    r.v[4] = hi.x; r.v[5] = hi.y; r.v[6] = hi.z; r.v[7] = hi.w;
    return r;
}
template <class T>
__device__ __forceinline__ void store32(T* p, const T& x) {
    uint4* q = reinterpret_cast<uint4*>(p);
    q[0] = make_uint4(x.v[0], x.v[1], x.v[2], x.v[3]);
    q[1] = make_uint4(x.v[4], x.v[5], x.v[6], x.v[7]);
}

}  // namespace g16d
