// BN254 G1 (over Fq) and G2 (over Fq2) point arithmetic for sm_100a.
//
// Buckets and running sums use XYZZ coordinates (x = X/ZZ, y = Y/ZZZ,
// ZZ^3 = ZZZ^2), the representation the reference's MSMs accumulate in
// (crates/msm/src/xyzz.rs; crates/cuda/src/kernels/bn254_curve.cuh:486-600).
// Formulas are the Explicit-Formulas Database ones for a = 0:
// madd-2008-s (8M + 2S), add-2008-s (12M + 2S), mdbl-2008-s-1 and
// dbl-2008-s-1.  ZZ = 0 is the identity.  The three exceptional cases of an
// incomplete addition (identity operand, P + P, P + (-P)) are handled
// explicitly: they are rare but reachable (duplicate bases, a bucket that
// cancels), and a wrong result there is a wrong proof.
//
// Affine inputs use the packed layout: x then y, Montgomery, with the point
// at infinity encoded as all-zero coordinates (gpu-layout/src/lib.rs:351).
#pragma once
#include "field.cuh"

namespace g16d {

template <class F>
struct Affine {
    F x, y;
    __device__ __forceinline__ bool is_inf() const { return x.is_zero() && y.is_zero(); }
};

template <class F>
struct Xyzz {
    F x, y, zz, zzz;
    __device__ __forceinline__ static Xyzz identity() {
        Xyzz r;
        r.x = F::one();
        r.y = F::one();
        r.zz = F::zero();
        r.zzz = F::zero();
        return r;
    }
    __device__ __forceinline__ bool is_inf() const { return zz.is_zero(); }
};

typedef Affine<Fq> G1Affine;
typedef Affine<Fq2> G2Affine;
typedef Xyzz<Fq> G1Xyzz;
typedef Xyzz<Fq2> G2Xyzz;

// The formulas below group independent products per dependency level
// (fmul2 / fmul3), which changes nothing in the values and lets the
// out-of-line variant (INL = false) overlap their carry chains.

// 2 * (x, y) for an affine point (mdbl-2008-s-1)
template <class F, bool INL = true>
__device__ __forceinline__ Xyzz<F> xyzz_dbl_affine(const F& x, const F& y) {
    F u = dbl(y);
    F v, xx, w, s, m2, t, wy;
    fmul2<INL>(u, u, x, x, v, xx);      // V = U^2, X^2
    fmul2<INL>(u, v, x, v, w, s);       // W = U V, S = X V
    F m = add(dbl(xx), xx);
    m2 = fsqr<INL>(m);
    Xyzz<F> r;
    r.x = sub(m2, dbl(s));
    fmul2<INL>(m, sub(s, r.x), w, y, t, wy);
    r.y = sub(t, wy);
    r.zz = v;
    r.zzz = w;
    return r;
}

// 2 * p (dbl-2008-s-1)
template <class F, bool INL = true>
__device__ __forceinline__ Xyzz<F> xyzz_dbl(const Xyzz<F>& p) {
    if (p.is_inf()) return p;
    F u = dbl(p.y);
    F v, xx, w, s, m2, t, wy;
    fmul2<INL>(u, u, p.x, p.x, v, xx);  // V = U^2, X^2
    fmul2<INL>(u, v, p.x, v, w, s);     // W = U V, S = X V
    F m = add(dbl(xx), xx);
    Xyzz<F> r;
    fmul2<INL>(m, m, v, p.zz, m2, r.zz);     // M^2, ZZ3 = V ZZ1
    r.x = sub(m2, dbl(s));
    fmul3<INL>(m, sub(s, r.x), w, p.y, w, p.zzz, t, wy, r.zzz);   // ZZZ3 = W ZZZ1
    r.y = sub(t, wy);
    return r;
}

// The doubling an addition falls into when both operands are equal: rare, so
// one out-of-line copy keeps it (and its call arguments) out of the hot loops.
template <class F>
__device__ __noinline__ Xyzz<F> xyzz_dbl_affine_ool(F x, F y) {
    return xyzz_dbl_affine<F, false>(x, y);
}
template <class F>
__device__ __noinline__ Xyzz<F> xyzz_dbl_ool(Xyzz<F> p) {
    return xyzz_dbl<F, false>(p);
}

// p + (x2, y2) for a finite affine point (madd-2008-s)
template <class F, bool INL = true>
__device__ __forceinline__ Xyzz<F> xyzz_add_affine(const Xyzz<F>& p, const F& x2, const F& y2) {
    if (p.is_inf()) {
        Xyzz<F> r;
        r.x = x2;
        r.y = y2;
        r.zz = F::one();
        r.zzz = F::one();
        return r;
    }
    F u2, s2;
    fmul2<INL>(x2, p.zz, y2, p.zzz, u2, s2);
    F pp_ = sub(u2, p.x);
    F rr = sub(s2, p.y);
    if (pp_.is_zero()) {
        if (rr.is_zero()) return xyzz_dbl_affine_ool<F>(x2, y2);   // rare: keep it out of the hot code
        return Xyzz<F>::identity();
    }
    Xyzz<F> r;
    if constexpr (INL) {
        // the accumulate kernel's inner loop: this order keeps the fewest
        // values live (registers bound its occupancy)
        F pp = sqr(pp_);
        F ppp = mul(pp_, pp);
        F q = mul(p.x, pp);
        r.x = sub(sub(sqr(rr), ppp), dbl(q));
        r.y = mul_sub(rr, sub(q, r.x), p.y, ppp);   // G1: one reduction for both products
        r.zz = mul(p.zz, pp);
        r.zzz = mul(p.zzz, ppp);
    } else {
        F pp, rr2, ppp, q, t, ypp;
        fmul2<INL>(pp_, pp_, rr, rr, pp, rr2);
        fmul2<INL>(pp_, pp, p.x, pp, ppp, q);
        r.x = sub(sub(rr2, ppp), dbl(q));
        fmul3<INL>(rr, sub(q, r.x), p.y, ppp, p.zzz, ppp, t, ypp, r.zzz);
        r.y = sub(t, ypp);
        r.zz = fmul<INL>(p.zz, pp);
    }
    return r;
}

// p + q (add-2008-s)
template <class F, bool INL = true>
__device__ __forceinline__ Xyzz<F> xyzz_add(const Xyzz<F>& p, const Xyzz<F>& q) {
    if (p.is_inf()) return q;
    if (q.is_inf()) return p;
    F u1, u2, s1, s2, zz12, zzz12;
    fmul3<INL>(p.x, q.zz, q.x, p.zz, p.zz, q.zz, u1, u2, zz12);
    fmul3<INL>(p.y, q.zzz, q.y, p.zzz, p.zzz, q.zzz, s1, s2, zzz12);
    F pp_ = sub(u2, u1);
    F rr = sub(s2, s1);
    if (pp_.is_zero()) {
        if (rr.is_zero()) return xyzz_dbl_ool<F>(p);   // rare: keep it out of the hot code
        return Xyzz<F>::identity();
    }
    F pp, rr2, ppp, qq, t, sppp;
    fmul2<INL>(pp_, pp_, rr, rr, pp, rr2);
    Xyzz<F> r;
    fmul3<INL>(pp_, pp, u1, pp, zz12, pp, ppp, qq, r.zz);
    r.x = sub(sub(rr2, ppp), dbl(qq));
    fmul3<INL>(rr, sub(qq, r.x), s1, ppp, zzz12, ppp, t, sppp, r.zzz);
    r.y = sub(t, sppp);
    return r;
}

// ---- global-memory codecs, 128-bit accesses ----
__device__ __forceinline__ Fq ld_fq(const uint4* p) {
    uint4 a = __ldg(p), b = __ldg(p + 1);
    Fq r;
    r.v[0] = a.x; r.v[1] = a.y; r.v[2] = a.z; r.v[3] = a.w;
    r.v[4] = b.x; r.v[5] = b.y; r.v[6] = b.z; r.v[7] = b.w;
    return r;
}
__device__ __forceinline__ void st_fq(uint4* p, const Fq& x) {
    p[0] = make_uint4(x.v[0], x.v[1], x.v[2], x.v[3]);
    p[1] = make_uint4(x.v[4], x.v[5], x.v[6], x.v[7]);
}
__device__ __forceinline__ Fq ld_fq_rw(const uint4* p) {
    uint4 a = p[0], b = p[1];
    Fq r;
    r.v[0] = a.x; r.v[1] = a.y; r.v[2] = a.z; r.v[3] = a.w;
    r.v[4] = b.x; r.v[5] = b.y; r.v[6] = b.z; r.v[7] = b.w;
    return r;
}

template <class F>
struct Codec;

template <>
struct Codec<Fq> {
    static constexpr int U4 = 2;   // uint4 per coordinate
    __device__ __forceinline__ static Fq ld(const uint4* p) { return ld_fq(p); }
    __device__ __forceinline__ static Fq ld_rw(const uint4* p) { return ld_fq_rw(p); }
    __device__ __forceinline__ static void st(uint4* p, const Fq& x) { st_fq(p, x); }
};

template <>
struct Codec<Fq2> {
    static constexpr int U4 = 4;
    __device__ __forceinline__ static Fq2 ld(const uint4* p) { return {ld_fq(p), ld_fq(p + 2)}; }
    __device__ __forceinline__ static Fq2 ld_rw(const uint4* p) { return {ld_fq_rw(p), ld_fq_rw(p + 2)}; }
    __device__ __forceinline__ static void st(uint4* p, const Fq2& x) {
        st_fq(p, x.c0);
        st_fq(p + 2, x.c1);
    }
};

template <class F>
__device__ __forceinline__ Affine<F> ld_affine(const uint4* base, size_t i) {
    constexpr int U = Codec<F>::U4;
    const uint4* p = base + i * (2 * U);
    return {Codec<F>::ld(p), Codec<F>::ld(p + U)};
}

// for memory the same kernel also writes (no read-only cache path)
template <class F>
__device__ __forceinline__ Affine<F> ld_affine_rw(const uint4* base, size_t i) {
    constexpr int U = Codec<F>::U4;
    const uint4* p = base + i * (2 * U);
    return {Codec<F>::ld_rw(p), Codec<F>::ld_rw(p + U)};
}

template <class F>
__device__ __forceinline__ void st_affine(uint4* base, size_t i, const F& x, const F& y) {
    constexpr int U = Codec<F>::U4;
    uint4* p = base + i * (2 * U);
    Codec<F>::st(p, x);
    Codec<F>::st(p + U, y);
}

template <class F>
__device__ __forceinline__ void st_xyzz(uint4* base, size_t i, const Xyzz<F>& x) {
    constexpr int U = Codec<F>::U4;
    uint4* p = base + i * (4 * U);
    Codec<F>::st(p, x.x);
    Codec<F>::st(p + U, x.y);
    Codec<F>::st(p + 2 * U, x.zz);
    Codec<F>::st(p + 3 * U, x.zzz);
}

template <class F>
__device__ __forceinline__ Xyzz<F> ld_xyzz(const uint4* base, size_t i) {
    constexpr int U = Codec<F>::U4;
    const uint4* p = base + i * (4 * U);
    return {Codec<F>::ld_rw(p), Codec<F>::ld_rw(p + U), Codec<F>::ld_rw(p + 2 * U), Codec<F>::ld_rw(p + 3 * U)};
}

}  // namespace g16d
