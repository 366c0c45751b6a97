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

// 2 * (x, y) for an affine point (mdbl-2008-s-1)
template <class F, bool INL = true>
__device__ __forceinline__ Xyzz<F> xyzz_dbl_affine(const F& x, const F& y) {
    F u = dbl(y);
    F v = fsqr<INL>(u);
    F w = fmul<INL>(u, v);
    F s = fmul<INL>(x, v);
    F xx = fsqr<INL>(x);
    F m = add(dbl(xx), xx);
    Xyzz<F> r;
    r.x = sub(fsqr<INL>(m), dbl(s));
    r.y = sub(fmul<INL>(m, sub(s, r.x)), fmul<INL>(w, y));
    r.zz = v;
    r.zzz = w;
    return r;
}

// 2 * p (dbl-2008-s-1)
template <class F, bool INL = true>
__device__ __forceinline__ Xyzz<F> xyzz_dbl(const Xyzz<F>& p) {
    if (p.is_inf()) return p;
    F u = dbl(p.y);
    F v = fsqr<INL>(u);
    F w = fmul<INL>(u, v);
    F s = fmul<INL>(p.x, v);
    F xx = fsqr<INL>(p.x);
    F m = add(dbl(xx), xx);
    Xyzz<F> r;
    r.x = sub(fsqr<INL>(m), dbl(s));
    r.y = sub(fmul<INL>(m, sub(s, r.x)), fmul<INL>(w, p.y));
    r.zz = fmul<INL>(v, p.zz);
    r.zzz = fmul<INL>(w, p.zzz);
    return r;
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
    F u2 = fmul<INL>(x2, p.zz);
    F s2 = fmul<INL>(y2, p.zzz);
    F pp_ = sub(u2, p.x);
    F rr = sub(s2, p.y);
    if (pp_.is_zero()) {
        if (rr.is_zero()) return xyzz_dbl_affine<F, false>(x2, y2);   // rare: keep it out of the hot code
        return Xyzz<F>::identity();
    }
    F pp = fsqr<INL>(pp_);
    F ppp = fmul<INL>(pp_, pp);
    F q = fmul<INL>(p.x, pp);
    Xyzz<F> r;
    r.x = sub(sub(fsqr<INL>(rr), ppp), dbl(q));
    r.y = sub(fmul<INL>(rr, sub(q, r.x)), fmul<INL>(p.y, ppp));
    r.zz = fmul<INL>(p.zz, pp);
    r.zzz = fmul<INL>(p.zzz, ppp);
    return r;
}

// p + q (add-2008-s)
template <class F, bool INL = true>
__device__ __forceinline__ Xyzz<F> xyzz_add(const Xyzz<F>& p, const Xyzz<F>& q) {
    if (p.is_inf()) return q;
    if (q.is_inf()) return p;
    F u1 = fmul<INL>(p.x, q.zz);
    F u2 = fmul<INL>(q.x, p.zz);
    F s1 = fmul<INL>(p.y, q.zzz);
    F s2 = fmul<INL>(q.y, p.zzz);
    F pp_ = sub(u2, u1);
    F rr = sub(s2, s1);
    if (pp_.is_zero()) {
        if (rr.is_zero()) return xyzz_dbl<F, false>(p);   // rare: keep it out of the hot code
        return Xyzz<F>::identity();
    }
    F pp = fsqr<INL>(pp_);
    F ppp = fmul<INL>(pp_, pp);
    F qq = fmul<INL>(u1, pp);
    Xyzz<F> r;
    r.x = sub(sub(fsqr<INL>(rr), ppp), dbl(qq));
    r.y = sub(fmul<INL>(rr, sub(qq, r.x)), fmul<INL>(s1, ppp));
    r.zz = fmul<INL>(fmul<INL>(p.zz, q.zz), pp);
    r.zzz = fmul<INL>(fmul<INL>(p.zzz, q.zzz), ppp);
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
