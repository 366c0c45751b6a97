// Host-side BN254 arithmetic for the library's control code: domain and
// twiddle tables, zkey decoding, the window combination after the device
// MSMs, stage-11 proof assembly and the synthetic key generator.
//
// 4 x u64 little-endian limbs, Montgomery form with R = 2^256, always fully
// reduced: bit-identical to arkworks' in-memory Fp and to the packed device
// layout (8 x u32 LE).  The hot path never runs here.
#pragma once
#include <cstdint>
#include <cstring>
#include <cstddef>

namespace g16 {

typedef unsigned __int128 u128;

struct Fe {
    uint64_t v[4];
};

struct FieldParams {
    uint64_t p[4];
    uint64_t n0;   // -p^-1 mod 2^64
    Fe one;        // R mod p
    Fe r2;         // R^2 mod p
};

// n0, R and R^2 from the modulus, at compile time: R mod p and R^2 mod p by
// 512 modular doublings of 1
constexpr FieldParams make_field(uint64_t p0, uint64_t p1, uint64_t p2, uint64_t p3) {
    FieldParams f{{p0, p1, p2, p3}, 0, {{0, 0, 0, 0}}, {{0, 0, 0, 0}}};
    uint64_t inv = 1;
    for (int i = 0; i < 7; i++) inv *= 2 - p0 * inv;
    f.n0 = (uint64_t)0 - inv;
    uint64_t x[4] = {1, 0, 0, 0};
    for (int i = 0; i < 512; i++) {
        if (i == 256)
            for (int j = 0; j < 4; j++) f.one.v[j] = x[j];
        uint64_t top = x[3] >> 63;
        for (int j = 3; j > 0; j--) x[j] = (x[j] << 1) | (x[j - 1] >> 63);
        x[0] <<= 1;
        bool ge = top != 0;
        if (!ge) {
            ge = true;   // equal counts as >=
            for (int j = 3; j >= 0; j--)
                if (x[j] != f.p[j]) {
                    ge = x[j] > f.p[j];
                    break;
                }
        }
        if (ge) {
            uint64_t br = 0;
            for (int j = 0; j < 4; j++) {
                uint64_t a = x[j], b = f.p[j];
                uint64_t d = a - b - br;
                br = (a < b || a - b < br) ? 1 : 0;
                x[j] = d;
            }
        }
    }
    for (int j = 0; j < 4; j++) f.r2.v[j] = x[j];
    return f;
}

inline constexpr FieldParams FR_P =
    make_field(0x43e1f593f0000001ULL, 0x2833e84879b97091ULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL);
inline constexpr FieldParams FQ_P =
    make_field(0x3c208c16d87cfd47ULL, 0x97816a916871ca8dULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL);
void host_init();

static inline bool geq4(const uint64_t* a, const uint64_t* p) {
    for (int i = 3; i >= 0; i--) {
        if (a[i] != p[i]) return a[i] > p[i];
    }
    return true;
}
static inline uint64_t sub4(uint64_t* r, const uint64_t* a, const uint64_t* b) {
    uint64_t br = 0;
    for (int i = 0; i < 4; i++) {
        u128 d = (u128)a[i] - b[i] - br;
        r[i] = (uint64_t)d;
        br = (uint64_t)(d >> 127);
    }
    return br;
}
static inline uint64_t add4(uint64_t* r, const uint64_t* a, const uint64_t* b) {
    uint64_t c = 0;
    for (int i = 0; i < 4; i++) {
        u128 s = (u128)a[i] + b[i] + c;
        r[i] = (uint64_t)s;
        c = (uint64_t)(s >> 64);
    }
    return c;
}

template <const FieldParams& P>
struct Fp {
    Fe x;
    static Fp zero() { Fp r; std::memset(&r, 0, sizeof r); return r; }
    static Fp one() { Fp r; r.x = P.one; return r; }
    static Fp raw(const uint64_t* v) { Fp r; std::memcpy(r.x.v, v, 32); return r; }
    bool is_zero() const { return (x.v[0] | x.v[1] | x.v[2] | x.v[3]) == 0; }
    bool operator==(const Fp& o) const { return std::memcmp(x.v, o.x.v, 32) == 0; }
    bool operator!=(const Fp& o) const { return !(*this == o); }
    // Branch-free: both moduli are below 2^254, so a sum of two reduced
    // values never carries out; the reduction is selected by a mask.
    Fp operator+(const Fp& o) const {
        Fp r;
        uint64_t s[4], d[4];
        add4(s, x.v, o.x.v);
        const uint64_t keep = (uint64_t)0 - sub4(d, s, P.p);   // all ones when s < p
        for (int i = 0; i < 4; i++) r.x.v[i] = (s[i] & keep) | (d[i] & ~keep);
        return r;
    }
    Fp operator-(const Fp& o) const {
        Fp r;
        uint64_t d[4], pm[4];
        const uint64_t mask = (uint64_t)0 - sub4(d, x.v, o.x.v);   // all ones on borrow
        for (int i = 0; i < 4; i++) pm[i] = P.p[i] & mask;
        add4(r.x.v, d, pm);
        return r;
    }
    Fp operator-() const { return is_zero() ? *this : zero() - *this; }
    Fp dbl() const { return *this + *this; }
    // CIOS Montgomery product, unrolled over the constant modulus.  Both BN254
    // moduli are below 2^254, so every partial result stays below 2p < 2^256
    // and no fifth word survives a round.
    Fp operator*(const Fp& o) const {
        const uint64_t* a = x.v;
        uint64_t t0 = 0, t1 = 0, t2 = 0, t3 = 0;
        for (int i = 0; i < 4; i++) {
            const uint64_t bi = o.x.v[i];
            u128 uv = (u128)a[0] * bi + t0;
            t0 = (uint64_t)uv;
            uint64_t c = (uint64_t)(uv >> 64);
            uv = (u128)a[1] * bi + t1 + c;
            t1 = (uint64_t)uv;
            c = (uint64_t)(uv >> 64);
            uv = (u128)a[2] * bi + t2 + c;
            t2 = (uint64_t)uv;
            c = (uint64_t)(uv >> 64);
            uv = (u128)a[3] * bi + t3 + c;
            t3 = (uint64_t)uv;
            const uint64_t t4 = (uint64_t)(uv >> 64);
            const uint64_t m = t0 * P.n0;
            uv = (u128)m * P.p[0] + t0;
            c = (uint64_t)(uv >> 64);
            uv = (u128)m * P.p[1] + t1 + c;
            t0 = (uint64_t)uv;
            c = (uint64_t)(uv >> 64);
            uv = (u128)m * P.p[2] + t2 + c;
            t1 = (uint64_t)uv;
            c = (uint64_t)(uv >> 64);
            uv = (u128)m * P.p[3] + t3 + c;
            t2 = (uint64_t)uv;
            t3 = t4 + (uint64_t)(uv >> 64);
        }
        Fp r;
        r.x.v[0] = t0;
        r.x.v[1] = t1;
        r.x.v[2] = t2;
        r.x.v[3] = t3;
        uint64_t d[4];
        if (!sub4(d, r.x.v, P.p)) std::memcpy(r.x.v, d, 32);
        return r;
    }
    Fp sqr() const { return *this * *this; }
    Fp pow(const uint64_t* e, int nlimbs) const {
        Fp acc = one(), b = *this;
        for (int i = nlimbs * 64 - 1; i >= 0; i--) {
            acc = acc.sqr();
            if ((e[i / 64] >> (i % 64)) & 1) acc = acc * b;
        }
        return acc;
    }
    Fp inv() const {
        uint64_t e[4], two[4] = {2, 0, 0, 0};
        sub4(e, P.p, two);
        return pow(e, 4);
    }
    // standard-form integer -> Montgomery
    static Fp from_std(const uint64_t* v) { Fp a = raw(v), r2; r2.x = P.r2; return a * r2; }
    static Fp from_u64(uint64_t v) { uint64_t t[4] = {v, 0, 0, 0}; return from_std(t); }
    // Montgomery -> standard-form integer
    void to_std(uint64_t* out) const {
        Fp one_raw = zero();
        one_raw.x.v[0] = 1;
        Fp r = *this * one_raw;
        std::memcpy(out, r.x.v, 32);
    }
    static bool canonical(const uint64_t* v) { return !geq4(v, P.p); }
};

typedef Fp<FR_P> Fr;
typedef Fp<FQ_P> Fq;

struct Fq2 {
    Fq c0, c1;
    static Fq2 zero() { return {Fq::zero(), Fq::zero()}; }
    static Fq2 one() { return {Fq::one(), Fq::zero()}; }
    bool is_zero() const { return c0.is_zero() && c1.is_zero(); }
    bool operator==(const Fq2& o) const { return c0 == o.c0 && c1 == o.c1; }
    Fq2 operator+(const Fq2& o) const { return {c0 + o.c0, c1 + o.c1}; }
    Fq2 operator-(const Fq2& o) const { return {c0 - o.c0, c1 - o.c1}; }
    Fq2 operator-() const { return {-c0, -c1}; }
    Fq2 dbl() const { return {c0.dbl(), c1.dbl()}; }
    Fq2 operator*(const Fq2& o) const {
        Fq t0 = c0 * o.c0, t1 = c1 * o.c1;
        Fq m = (c0 + c1) * (o.c0 + o.c1);
        return {t0 - t1, m - t0 - t1};
    }
    Fq2 sqr() const { return *this * *this; }
    Fq2 inv() const {
        Fq n = (c0.sqr() + c1.sqr()).inv();
        return {c0 * n, -(c1 * n)};
    }
};

// ---- short Weierstrass points, a = 0; Jacobian with Z = 0 as infinity ----
template <class F>
struct Affine {
    F x, y;
    bool inf;
};

template <class F>
struct Jac {
    F x, y, z;
    static Jac identity() { Jac r; r.x = F::one(); r.y = F::one(); r.z = F::zero(); return r; }
    bool is_inf() const { return z.is_zero(); }
    static Jac from_affine(const Affine<F>& a) {
        if (a.inf) return identity();
        Jac r;
        r.x = a.x;
        r.y = a.y;
        r.z = F::one();
        return r;
    }
    Jac dbl() const {
        if (is_inf()) return *this;
        F A = x.sqr(), B = y.sqr(), C = B.sqr();
        F D = ((x + B).sqr() - A - C).dbl();
        F E = A.dbl() + A;
        F Fv = E.sqr();
        Jac r;
        r.x = Fv - D.dbl();
        r.y = E * (D - r.x) - C.dbl().dbl().dbl();
        r.z = (y * z).dbl();
        return r;
    }
    Jac operator+(const Jac& q) const {
        if (is_inf()) return q;
        if (q.is_inf()) return *this;
        F z1z1 = z.sqr(), z2z2 = q.z.sqr();
        F u1 = x * z2z2, u2 = q.x * z1z1;
        F s1 = y * q.z * z2z2, s2 = q.y * z * z1z1;
        F h = u2 - u1, rr = s2 - s1;
        if (h.is_zero()) return rr.is_zero() ? dbl() : identity();
        F i = h.dbl().sqr(), j = h * i;
        rr = rr.dbl();
        F v = u1 * i;
        Jac r;
        r.x = rr.sqr() - j - v.dbl();
        r.y = rr * (v - r.x) - (s1 * j).dbl();
        r.z = ((z + q.z).sqr() - z1z1 - z2z2) * h;
        return r;
    }
    Jac add_affine(const Affine<F>& q) const {
        if (q.inf) return *this;
        if (is_inf()) return from_affine(q);
        F z1z1 = z.sqr();
        F u2 = q.x * z1z1, s2 = q.y * z * z1z1;
        F h = u2 - x, rr = s2 - y;
        if (h.is_zero()) return rr.is_zero() ? dbl() : identity();
        F hh = h.sqr(), i = hh.dbl().dbl(), j = h * i;
        rr = rr.dbl();
        F v = x * i;
        Jac r;
        r.x = rr.sqr() - j - v.dbl();
        r.y = rr * (v - r.x) - (y * j).dbl();
        r.z = (z + h).sqr() - z1z1 - hh;
        return r;
    }
    Jac neg() const { Jac r = *this; r.y = -y; return r; }
    // scalar in standard form (4 limbs)
    Jac mul(const uint64_t* k) const {
        Jac acc = identity();
        for (int i = 255; i >= 0; i--) {
            acc = acc.dbl();
            if ((k[i / 64] >> (i % 64)) & 1) acc = acc + *this;
        }
        return acc;
    }
    Affine<F> to_affine() const {
        Affine<F> a;
        if (is_inf()) { a.x = F::zero(); a.y = F::zero(); a.inf = true; return a; }
        F zi = z.inv(), zi2 = zi.sqr();
        a.x = x * zi2;
        a.y = y * zi2 * zi;
        a.inf = false;
        return a;
    }
};

typedef Affine<Fq> G1A;
typedef Affine<Fq2> G2A;
typedef Jac<Fq> G1J;
typedef Jac<Fq2> G2J;

extern G1A G1_GENERATOR;
extern G2A G2_GENERATOR;
extern Fq2 TWIST_B;   // 3 / (9 + u)

// ---- packed byte layout: Montgomery LE coordinates, infinity = all zero ----
inline void pack(uint8_t* out, const G1A& p) {
    if (p.inf) { std::memset(out, 0, 64); return; }
    std::memcpy(out, p.x.x.v, 32);
    std::memcpy(out + 32, p.y.x.v, 32);
}
inline void pack(uint8_t* out, const G2A& p) {
    if (p.inf) { std::memset(out, 0, 128); return; }
    std::memcpy(out, p.x.c0.x.v, 32);
    std::memcpy(out + 32, p.x.c1.x.v, 32);
    std::memcpy(out + 64, p.y.c0.x.v, 32);
    std::memcpy(out + 96, p.y.c1.x.v, 32);
}
// false when a coordinate is not below q
inline bool unpack(G1A& p, const uint8_t* in) {
    uint64_t v[2][4];
    std::memcpy(v, in, 64);
    if (!Fq::canonical(v[0]) || !Fq::canonical(v[1])) return false;
    p.x = Fq::raw(v[0]);
    p.y = Fq::raw(v[1]);
    p.inf = p.x.is_zero() && p.y.is_zero();
    return true;
}
inline bool unpack(G2A& p, const uint8_t* in) {
    uint64_t v[4][4];
    std::memcpy(v, in, 128);
    for (int i = 0; i < 4; i++)
        if (!Fq::canonical(v[i])) return false;
    p.x = {Fq::raw(v[0]), Fq::raw(v[1])};
    p.y = {Fq::raw(v[2]), Fq::raw(v[3])};
    p.inf = p.x.is_zero() && p.y.is_zero();
    return true;
}

template <class F>
inline bool on_curve(const Affine<F>& p);
template <>
inline bool on_curve(const G1A& p) {
    if (p.inf) return true;
    return p.y.sqr() == p.x.sqr() * p.x + Fq::from_u64(3);
}
template <>
inline bool on_curve(const G2A& p) {
    if (p.inf) return true;
    return p.y.sqr() == p.x.sqr() * p.x + TWIST_B;
}

// omega_n for n = 2^log_n: 5^((r-1)/2^28) squared (28 - log_n) times
Fr domain_root(int log_n);

// batch-normalise Jacobian points to affine with one inversion
template <class F>
void batch_to_affine(const Jac<F>* in, Affine<F>* out, size_t n);

}  // namespace g16
