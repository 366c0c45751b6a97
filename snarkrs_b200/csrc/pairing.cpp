// Host optimal-ate pairing and Groth16 verifier (see pairing.hpp).
//
// Miller loop: homogeneous projective coordinates on the twist, so no
// inversion per step.  With T = (X : Y : Z) and a slope N/D the line through
// the untwisted points, evaluated at P = (xP, yP) and multiplied by an element
// of Fq2 (which the final exponentiation removes), is
//     D*Z*yP  -  N*Z*xP * w  +  (N*X - D*Y) * w^3            (tangent at T)
//     D*yP    -  N*xP * w    +  (N*xQ - D*yQ) * w^3          (chord T, Q)
// and the doubled / added point follows from the affine formulas with
// Z' = D^3 * Z.  The loop runs over the binary digits of 6u + 2 and ends with
// the two Frobenius-twisted additions of the optimal ate pairing (Vercauteren,
// "Optimal pairings", 2010).
//
// Final exponentiation: (p^6 - 1)(p^2 + 1) by conjugation, one inversion and a
// Frobenius; the hard part (p^4 - p^2 + 1)/r by the vectorial addition chain
// of Scott, Benger, Charlemagne, Dominguez Perez and Kachisa, "On the final
// exponentiation for calculating pairings on ordinary elliptic curves" (2009),
// with three exponentiations by u.  Frobenius constants are computed at start
// up as powers of xi.
#include "pairing.hpp"
#include <future>
#include <mutex>
#include <vector>

namespace g16 {

namespace {

const uint64_t BN_U = 4965661367192848881ULL;   // the BN parameter u of BN254

// ---------------------------------------------------------------- towers
Fq2 fq2_mul_fq(const Fq2& a, const Fq& s) { return {a.c0 * s, a.c1 * s}; }
Fq2 fq2_conj(const Fq2& a) { return {a.c0, -a.c1}; }
// (a + b u)(9 + u) = (9a - b) + (a + 9b) u
Fq2 mul_xi(const Fq2& a) {
    Fq a2 = a.c0.dbl(), a4 = a2.dbl(), a8 = a4.dbl();
    Fq b2 = a.c1.dbl(), b4 = b2.dbl(), b8 = b4.dbl();
    return {a8 + a.c0 - a.c1, a.c0 + b8 + a.c1};
}

struct Fq6 {
    Fq2 c0, c1, c2;
    static Fq6 zero() { return {Fq2::zero(), Fq2::zero(), Fq2::zero()}; }
    static Fq6 one() { return {Fq2::one(), Fq2::zero(), Fq2::zero()}; }
    bool is_zero() const { return c0.is_zero() && c1.is_zero() && c2.is_zero(); }
    bool operator==(const Fq6& o) const { return c0 == o.c0 && c1 == o.c1 && c2 == o.c2; }
    Fq6 operator+(const Fq6& o) const { return {c0 + o.c0, c1 + o.c1, c2 + o.c2}; }
    Fq6 operator-(const Fq6& o) const { return {c0 - o.c0, c1 - o.c1, c2 - o.c2}; }
    Fq6 operator-() const { return {-c0, -c1, -c2}; }
    // schoolbook with v^3 = xi, Karatsuba on the cross terms
    Fq6 operator*(const Fq6& o) const {
        Fq2 t0 = c0 * o.c0, t1 = c1 * o.c1, t2 = c2 * o.c2;
        Fq2 s12 = (c1 + c2) * (o.c1 + o.c2) - t1 - t2;   // c1 o2 + c2 o1
        Fq2 s01 = (c0 + c1) * (o.c0 + o.c1) - t0 - t1;   // c0 o1 + c1 o0
        Fq2 s02 = (c0 + c2) * (o.c0 + o.c2) - t0 - t2;   // c0 o2 + c2 o0
        return {t0 + mul_xi(s12), s01 + mul_xi(t2), s02 + t1};
    }
    Fq6 mul_v() const { return {mul_xi(c2), c0, c1}; }
    Fq6 inv() const {
        Fq2 t0 = c0.sqr() - mul_xi(c1 * c2);
        Fq2 t1 = mul_xi(c2.sqr()) - c0 * c1;
        Fq2 t2 = c1.sqr() - c0 * c2;
        Fq2 nrm = c0 * t0 + mul_xi(c2 * t1 + c1 * t2);
        Fq2 ni = nrm.inv();
        return {t0 * ni, t1 * ni, t2 * ni};
    }
};

struct Fq12 {
    Fq6 c0, c1;
    static Fq12 one() { return {Fq6::one(), Fq6::zero()}; }
    bool is_one() const { return c0 == Fq6::one() && c1.is_zero(); }
    Fq12 operator*(const Fq12& o) const {
        Fq6 t0 = c0 * o.c0, t1 = c1 * o.c1;
        Fq6 m = (c0 + c1) * (o.c0 + o.c1) - t0 - t1;
        return {t0 + t1.mul_v(), m};
    }
    // (a0 + a1 w)^2 = a0^2 + a1^2 v + 2 a0 a1 w, with two Fq6 products:
    // a0^2 + a1^2 v = (a0 + a1)(a0 + a1 v) - t - t v for t = a0 a1
    Fq12 sqr() const {
        Fq6 t = c0 * c1;
        Fq6 m = (c0 + c1) * (c0 + c1.mul_v());
        return {m - t - t.mul_v(), t + t};
    }
    Fq12 conj() const { return {c0, -c1}; }
    Fq12 inv() const {
        Fq6 d = (c0 * c0 - (c1 * c1).mul_v()).inv();
        return {c0 * d, -(c1 * d)};
    }
};

// ---------------------------------------------------------------- constants
// little-endian multi-limb integers for the Frobenius exponents
typedef std::vector<uint64_t> Big;

Big big_mul(const Big& a, const Big& b) {
    Big r(a.size() + b.size(), 0);
    for (size_t i = 0; i < a.size(); i++) {
        u128 c = 0;
        for (size_t j = 0; j < b.size(); j++) {
            u128 t = (u128)a[i] * b[j] + r[i + j] + c;
            r[i + j] = (uint64_t)t;
            c = t >> 64;
        }
        r[i + b.size()] = (uint64_t)c;
    }
    return r;
}

// (a - 1) / d for a = 1 mod d
Big big_dec_div(Big a, uint64_t d) {
    for (size_t i = 0; i < a.size(); i++) {
        if (a[i]--) break;
    }
    u128 rem = 0;
    for (size_t i = a.size(); i-- > 0;) {
        u128 cur = (rem << 64) | a[i];
        a[i] = (uint64_t)(cur / d);
        rem = cur % d;
    }
    return a;
}

Fq2 fq2_pow(const Fq2& b, const Big& e) {
    Fq2 acc = Fq2::one();
    for (size_t i = e.size() * 64; i-- > 0;) {
        acc = acc.sqr();
        if ((e[i / 64] >> (i % 64)) & 1) acc = acc * b;
    }
    return acc;
}

struct Consts {
    Fq2 gamma[4][6];   // gamma[k][j] = xi^(j (p^k - 1) / 6), k = 1, 2, 3
    uint64_t r_std[4];
};

const Consts& consts() {
    static Consts K;
    static std::once_flag once;
    std::call_once(once, [] {
        host_init();
        Big p(FQ_P.p, FQ_P.p + 4);
        Big pk = p;
        Fq2 xi = {Fq::from_u64(9), Fq::one()};
        for (int k = 1; k <= 3; k++) {
            Fq2 g = fq2_pow(xi, big_dec_div(pk, 6));   // xi^((p^k - 1) / 6)
            K.gamma[k][0] = Fq2::one();
            for (int j = 1; j < 6; j++) K.gamma[k][j] = K.gamma[k][j - 1] * g;
            pk = big_mul(pk, p);
        }
        for (int i = 0; i < 4; i++) K.r_std[i] = FR_P.p[i];
    });
    return K;
}

// f^(p^k) for k = 1, 2, 3: with f = sum_j b_j w^j, b_j in Fq2,
// f^(p^k) = sum_j conj^k(b_j) gamma_k^j w^j.
Fq12 frobenius(const Fq12& f, int k) {
    const Consts& K = consts();
    Fq2 b[6] = {f.c0.c0, f.c1.c0, f.c0.c1, f.c1.c1, f.c0.c2, f.c1.c2};   // w^0 .. w^5
    for (int j = 0; j < 6; j++) {
        if (k & 1) b[j] = fq2_conj(b[j]);
        b[j] = b[j] * K.gamma[k][j];
    }
    return {{b[0], b[2], b[4]}, {b[1], b[3], b[5]}};
}

// ---------------------------------------------------------------- Miller loop
struct Proj {
    Fq2 x, y, z;
};

// sparse line c0 = (l0, 0, 0), c1 = (l1, l3, 0): l0 + l1 w + l3 w^3
struct Line {
    Fq2 l0, l1, l3;
};

// a * (b0 + b1 v) for b with no v^2 term
Fq6 mul_by_01(const Fq6& a, const Fq2& b0, const Fq2& b1) {
    Fq2 t0 = a.c0 * b0, t1 = a.c1 * b1;
    Fq2 x0 = mul_xi((a.c1 + a.c2) * b1 - t1) + t0;   // a0 b0 + xi a2 b1
    Fq2 x1 = (a.c0 + a.c1) * (b0 + b1) - t0 - t1;    // a0 b1 + a1 b0
    Fq2 x2 = (a.c0 + a.c2) * b0 - t0 + t1;           // a2 b0 + a1 b1
    return {x0, x1, x2};
}

// f * (L0 + L1 w) with L0 = (l0, 0, 0) and L1 = (l1, l3, 0)
Fq12 mul_line(const Fq12& f, const Line& l) {
    Fq6 t0 = {f.c0.c0 * l.l0, f.c0.c1 * l.l0, f.c0.c2 * l.l0};
    Fq6 t1 = mul_by_01(f.c1, l.l1, l.l3);
    Fq6 m = mul_by_01(f.c0 + f.c1, l.l0 + l.l1, l.l3);
    return {t0 + t1.mul_v(), m - t0 - t1};
}

Line dbl_step(Proj& t, const G1A& p) {
    Fq2 xx = t.x.sqr();
    Fq2 n = xx.dbl() + xx;            // 3 X^2
    Fq2 d = (t.y * t.z).dbl();        // 2 Y Z
    Line l;
    l.l0 = fq2_mul_fq(d * t.z, p.y);
    l.l1 = -fq2_mul_fq(n * t.z, p.x);
    l.l3 = n * t.x - d * t.y;
    Fq2 d2 = d.sqr(), d3 = d2 * d, n2z = n.sqr() * t.z, xd2 = t.x * d2;
    Proj r;
    r.x = d * (n2z - xd2.dbl());
    r.y = n * (xd2.dbl() + xd2 - n2z) - t.y * d3;
    r.z = d3 * t.z;
    t = r;
    return l;
}

Line add_step(Proj& t, const G2A& q, const G1A& p) {
    Fq2 n = q.y * t.z - t.y;
    Fq2 d = q.x * t.z - t.x;
    Line l;
    l.l0 = fq2_mul_fq(d, p.y);
    l.l1 = -fq2_mul_fq(n, p.x);
    l.l3 = n * q.x - d * q.y;
    Fq2 d2 = d.sqr(), d3 = d2 * d, n2z = n.sqr() * t.z;
    Proj r;
    r.x = d * (n2z - d2 * (t.x + q.x * t.z));
    r.y = n * (d2 * (t.x.dbl() + q.x * t.z) - n2z) - t.y * d3;
    r.z = d3 * t.z;
    t = r;
    return l;
}

// pi(Q) and -pi^2(Q) on the twist
G2A twist_frob(const G2A& q) {
    const Consts& K = consts();
    return {fq2_conj(q.x) * K.gamma[1][2], fq2_conj(q.y) * K.gamma[1][3], q.inf};
}
G2A twist_frob2_neg(const G2A& q) {
    const Consts& K = consts();
    return {q.x * K.gamma[2][2], -(q.y * K.gamma[2][3]), q.inf};
}

Fq12 miller_loop(const G1A* ps, const G2A* qs, size_t n) {
    // 6u + 2 as a 65-bit number: hi bit 64 plus the low word
    const u128 s = (u128)BN_U * 6 + 2;
    int top = 127;
    while (!((s >> top) & 1)) top--;
    std::vector<Proj> t;
    std::vector<size_t> live;
    for (size_t i = 0; i < n; i++)
        if (!ps[i].inf && !qs[i].inf) {
            live.push_back(i);
            t.push_back({qs[i].x, qs[i].y, Fq2::one()});
        }
    Fq12 f = Fq12::one();
    for (int bit = top - 1; bit >= 0; bit--) {
        f = f.sqr();
        for (size_t k = 0; k < live.size(); k++) f = mul_line(f, dbl_step(t[k], ps[live[k]]));
        if ((s >> bit) & 1)
            for (size_t k = 0; k < live.size(); k++) f = mul_line(f, add_step(t[k], qs[live[k]], ps[live[k]]));
    }
    for (size_t k = 0; k < live.size(); k++) {
        const G1A& p = ps[live[k]];
        G2A q1 = twist_frob(qs[live[k]]), q2 = twist_frob2_neg(qs[live[k]]);
        f = mul_line(f, add_step(t[k], q1, p));
        f = mul_line(f, add_step(t[k], q2, p));
    }
    return f;
}

// ---------------------------------------------------------------- final exponentiation
// Squaring in the cyclotomic subgroup (Granger and Scott, "Faster squaring in
// the cyclotomic subgroup of sixth degree extensions", PKC 2010).  With
// t = w^3 (t^2 = xi), Fq12 = Fq4[w]/(w^3 - t) over Fq4 = Fq2[t], and
// f = A + B w + C w^2 whose coefficients are, in powers of w,
// A = b0 + b3 t, B = b1 + b4 t, C = b2 + b5 t.  For f with f^(p^6 + 1) = 1:
//   f^2 = (3 A^2 - 2 conj(A)) + (3 t C^2 + 2 conj(B)) w + (3 B^2 - 2 conj(C)) w^2,
// conj being t -> -t.  Each Fq4 square costs three Fq2 squarings.
void fq4_sqr(const Fq2& x0, const Fq2& x1, Fq2& y0, Fq2& y1) {
    Fq2 a = x0.sqr(), b = x1.sqr();
    y0 = a + mul_xi(b);
    y1 = (x0 + x1).sqr() - a - b;
}

Fq12 cyclotomic_sqr(const Fq12& f) {
    Fq2 b0 = f.c0.c0, b1 = f.c1.c0, b2 = f.c0.c1, b3 = f.c1.c1, b4 = f.c0.c2, b5 = f.c1.c2;
    Fq2 a0, a1, s0, s1, c0, c1;
    fq4_sqr(b0, b3, a0, a1);   // A^2
    fq4_sqr(b1, b4, s0, s1);   // B^2
    fq4_sqr(b2, b5, c0, c1);   // C^2
    // 3 x - 2 y = 2 (x - y) + x and 3 x + 2 y = 2 (x + y) + x
    Fq2 na0 = (a0 - b0).dbl() + a0, na1 = (a1 + b3).dbl() + a1;
    Fq2 tc0 = mul_xi(c1);                    // t C^2 = xi c1 + c0 t
    Fq2 nb0 = (tc0 + b1).dbl() + tc0, nb1 = (c0 - b4).dbl() + c0;
    Fq2 nc0 = (s0 - b2).dbl() + s0, nc1 = (s1 + b5).dbl() + s1;
    // back to powers of w: A -> (w^0, w^3), B -> (w^1, w^4), C -> (w^2, w^5)
    return {{na0, nc0, nb1}, {nb0, na1, nc1}};
}

// f^u for f in the cyclotomic subgroup (u > 0, so no conjugation)
Fq12 exp_u(const Fq12& f) {
    Fq12 acc = Fq12::one();
    for (int i = 63; i >= 0; i--) {
        acc = cyclotomic_sqr(acc);
        if ((BN_U >> i) & 1) acc = acc * f;
    }
    return acc;
}

Fq12 final_exponentiation(const Fq12& m) {
    // easy part: m^((p^6 - 1)(p^2 + 1))
    Fq12 f = m.conj() * m.inv();
    f = frobenius(f, 2) * f;
    // hard part: f^(lambda_0 + lambda_1 p + lambda_2 p^2 + lambda_3 p^3); in the
    // cyclotomic subgroup an inverse is a conjugate
    Fq12 fu = exp_u(f), fu2 = exp_u(fu), fu3 = exp_u(fu2);
    Fq12 y0 = frobenius(f, 1) * frobenius(f, 2) * frobenius(f, 3);
    Fq12 y1 = f.conj();
    Fq12 y2 = frobenius(fu2, 2);
    Fq12 y3 = frobenius(fu, 1).conj();
    Fq12 y4 = (fu * frobenius(fu2, 1)).conj();
    Fq12 y5 = fu2.conj();
    Fq12 y6 = (fu3 * frobenius(fu3, 1)).conj();
    Fq12 t0 = y6.sqr() * y4 * y5;
    Fq12 t1 = y3 * y5 * t0;
    t0 = t0 * y2;
    t1 = (t1.sqr() * t0).sqr();
    t0 = t1 * y1;
    t1 = t1 * y0;
    return t0.sqr() * t1;
}

bool in_g2_subgroup(const G2A& q) {
    if (q.inf) return true;
    return G2J::from_affine(q).mul(consts().r_std).is_inf();
}

// sum_i k_i P_i for a few points (Straus: 4-bit windows, shared doublings,
// per-point tables of 1..15 P_i normalised to affine together)
G1J small_msm(const G1A* pts, const uint64_t (*k)[4], size_t n) {
    std::vector<G1J> jt(n * 15);
    for (size_t i = 0; i < n; i++) {
        G1J p = G1J::from_affine(pts[i]);
        jt[i * 15] = p;
        for (int j = 1; j < 15; j++) jt[i * 15 + j] = jt[i * 15 + j - 1] + p;
    }
    std::vector<G1A> tab(n * 15);
    batch_to_affine(jt.data(), tab.data(), jt.size());
    G1J acc = G1J::identity();
    for (int w = 63; w >= 0; w--) {
        for (int d = 0; d < 4; d++) acc = acc.dbl();
        for (size_t i = 0; i < n; i++) {
            unsigned dg = (unsigned)(k[i][w / 16] >> (4 * (w % 16))) & 15u;
            if (dg) acc = acc.add_affine(tab[i * 15 + dg - 1]);
        }
    }
    return acc;
}

// the Miller loops of the pairs in parallel (their product is the Miller
// value of all pairs), then one final exponentiation
bool product_is_one(const G1A* p, const G2A* q, size_t n) {
    std::vector<std::future<Fq12>> parts;
    for (size_t i = 1; i < n; i++)
        parts.push_back(std::async(std::launch::async, [p, q, i] { return miller_loop(p + i, q + i, 1); }));
    Fq12 f = n ? miller_loop(p, q, 1) : Fq12::one();
    for (auto& x : parts) f = f * x.get();
    return final_exponentiation(f).is_one();
}

}  // namespace

bool pairing_product_is_one(const G1A* p, const G2A* q, size_t n) {
    consts();
    return product_is_one(p, q, n);
}

VerifyResult groth16_verify(const VerifyingKey& vk, const uint8_t* public_mont, size_t n_public, const G1A& a,
                            const G2A& b, const G1A& c, std::string* why) {
    auto say = [&](const char* s) {
        if (why) *why = s;
    };
    consts();
    // VerifyingKey::check_structure (crates/formats/src/lib.rs:1326-1345)
    if (vk.alpha1.inf || vk.beta2.inf || vk.gamma2.inf || vk.delta2.inf) {
        say("a verifying-key point is the point at infinity");
        return VerifyResult::UnsafeKey;
    }
    if (vk.gamma2.x == vk.delta2.x && vk.gamma2.y == vk.delta2.y) {
        say("gamma_g2 equals delta_g2: the key had no phase-2 contribution");
        return VerifyResult::UnsafeKey;
    }
    // check_proof (crates/groth16/src/verify.rs:80-108)
    if (a.inf || b.inf || c.inf) {
        say(a.inf ? "A is the point at infinity" : b.inf ? "B is the point at infinity" : "C is the point at infinity");
        return VerifyResult::InvalidProof;
    }
    if (!on_curve(a)) {
        say("A is not a valid G1 point");
        return VerifyResult::InvalidProof;
    }
    if (!on_curve(c)) {
        say("C is not a valid G1 point");
        return VerifyResult::InvalidProof;
    }
    if (!on_curve(b)) {
        say("B is not a valid G2 point");
        return VerifyResult::InvalidProof;
    }
    // B's subgroup check runs beside the pairing; an invalid B is refused
    // whatever the pairing says (crates/groth16/src/verify.rs:57-66)
    auto b_ok = std::async(std::launch::async, [&b] { return in_g2_subgroup(b); });
    // aggregate_public (crates/groth16/src/verify.rs:150-175)
    if (vk.n_ic == 0) {
        say("verifying key has an empty IC");
        b_ok.wait();
        return VerifyResult::EmptyKey;
    }
    if (n_public != vk.n_ic - 1) {
        say("public input count does not match the key");
        b_ok.wait();
        return VerifyResult::PublicInputCount;
    }
    std::vector<uint64_t[4]> k(n_public);
    for (size_t i = 0; i < n_public; i++) {
        uint64_t v[4];
        std::memcpy(v, public_mont + 32 * i, 32);
        Fr::raw(v).to_std(k[i]);
    }
    G1J l = G1J::from_affine(vk.ic[0]) + small_msm(vk.ic + 1, k.data(), n_public);
    G1A lbar = l.to_affine();
    G1A neg_a = a;
    neg_a.y = -a.y;
    G1A ps[4] = {neg_a, vk.alpha1, lbar, c};
    G2A qs[4] = {b, vk.beta2, vk.gamma2, vk.delta2};
    bool paired = product_is_one(ps, qs, 4);
    if (!b_ok.get()) {
        say("B is not a valid G2 point");
        return VerifyResult::InvalidProof;
    }
    if (!paired) {
        say("pairing check failed");
        return VerifyResult::PairingFailed;
    }
    return VerifyResult::Ok;
}

}  // namespace g16
