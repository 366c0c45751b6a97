// gnark v0.14 Groth16 BN254 files on the host: the proving-key dump
// (ProvingKey.WriteDump), the verifying key (VerifyingKey.WriteTo or
// WriteRawTo) and the witness dump of W, A.w and B.w -- the reference's
// crates/gnark (pk.rs, vk.rs, witness.rs).  The key is read into the same
// ZkeyHost the .zkey reader fills, with gnark's H basis: G1.Z holds n - 1 bases
// for H's coefficients in bit-reversed order, and the key has no constraint
// matrices, so it proves only from A.w and B.w rows.
//
// Two encodings meet in these files.  Encoder points (the dump's five header
// points, the verifying key) are canonical big-endian coordinates, X then Y,
// G2 as A1 before A0, with a flag in the top two bits of the first byte: 00
// uncompressed, 01 compressed infinity, 10 / 11 compressed with the smaller /
// larger Y (larger: above (q - 1) / 2; for Fq2 decided by A1 unless it is zero,
// then by A0).  Dumped slices are a u64 little-endian count and the elements'
// memory: Montgomery limbs, little-endian, G2 coordinates A0 before A1 -- the
// packed layout of this library, so they are copied as they are.
#include <cstring>
#include <string>
#include <vector>
#include "common.cuh"
#include "formats.hpp"
#include "host_bn254.hpp"

namespace g16 {

namespace {

struct Reader {
    const uint8_t* d;
    size_t len, pos = 0;
    const char* part = "";
    bool ok = true;

    const uint8_t* take(size_t n) {
        if (!ok) return nullptr;
        if (n > len - pos) {
            set_error("gnark %s: wanted %zu bytes at offset %zu, only %zu left", part, n, pos, len - pos);
            ok = false;
            return nullptr;
        }
        const uint8_t* p = d + pos;
        pos += n;
        return p;
    }
    bool be(size_t n, uint64_t& v) {
        const uint8_t* b = take(n);
        if (!b) return false;
        v = 0;
        for (size_t i = 0; i < n; i++) v = (v << 8) | b[i];
        return true;
    }
    bool le64(uint64_t& v) {
        const uint8_t* b = take(8);
        if (!b) return false;
        std::memcpy(&v, b, 8);
        return true;
    }
    // a dumped slice: u64 LE count, then count records of stride bytes
    const uint8_t* dumped(size_t stride, size_t& count) {
        uint64_t n = 0;
        if (!le64(n)) return nullptr;
        if (n > (len - pos) / stride) {
            set_error("gnark %s: %llu records of %zu bytes, only %zu bytes left", part, (unsigned long long)n, stride,
                      len - pos);
            ok = false;
            return nullptr;
        }
        count = (size_t)n;
        return take(count * stride);
    }
    bool fail(const char* what) {
        set_error("gnark %s: %s", part, what);
        ok = false;
        return false;
    }
};

// 32 big-endian bytes -> standard-form limbs; false at or above the modulus
template <class F>
bool be_elem(const uint8_t* b, F& out) {
    uint64_t v[4];
    for (int l = 0; l < 4; l++) {
        uint64_t x = 0;
        for (int i = 0; i < 8; i++) x = (x << 8) | b[(3 - l) * 8 + i];
        v[l] = x;
    }
    if (!F::canonical(v)) return false;
    out = F::from_std(v);
    return true;
}

// (q - 1) / 2 < y as integers
bool fq_larger(const Fq& y) {
    uint64_t v[4], half[4];
    y.to_std(v);
    for (int l = 0; l < 4; l++) half[l] = (FQ_P.p[l] >> 1) | (l < 3 ? FQ_P.p[l + 1] << 63 : 0);
    for (int l = 3; l >= 0; l--)
        if (v[l] != half[l]) return v[l] > half[l];
    return false;
}

// q = 3 mod 4: sqrt(a) = a^((q + 1) / 4) when a is a square
bool fq_sqrt(const Fq& a, Fq& out) {
    uint64_t e[4];
    uint64_t carry = 1;   // (q + 1) / 4 = ((q + 1) >> 2)
    for (int l = 0; l < 4; l++) {
        const uint64_t s = FQ_P.p[l] + carry;
        carry = s < carry ? 1 : 0;
        e[l] = s;
    }
    for (int l = 0; l < 4; l++) e[l] = (e[l] >> 2) | (l < 3 ? e[l + 1] << 62 : 0);
    out = a.pow(e, 4);
    return out.sqr() == a;
}

// Fq2 square root for q = 3 mod 4 (Adj and Rodriguez-Henriquez 2012,
// Algorithm 9): a1 = a^((q - 3) / 4), x0 = a1 a, alpha = a1 x0; alpha = -1
// gives x = u x0, else x = (1 + alpha)^((q - 1) / 2) x0.
bool fq2_sqrt(const Fq2& a, Fq2& out) {
    if (a.is_zero()) {
        out = a;
        return true;
    }
    // the exponents over Fq2 need the field's limbs: powers by square and multiply
    auto pw = [](Fq2 b, const uint64_t* e) {
        Fq2 acc = Fq2::one();
        for (int i = 255; i >= 0; i--) {
            acc = acc.sqr();
            if ((e[i / 64] >> (i % 64)) & 1) acc = acc * b;
        }
        return acc;
    };
    uint64_t e1[4], e2[4];
    {   // (q - 3) / 4 and (q - 1) / 2
        uint64_t borrow = 3, t[4];
        for (int l = 0; l < 4; l++) {
            const uint64_t p = FQ_P.p[l];
            t[l] = p - borrow;
            borrow = p < borrow ? 1 : 0;
        }
        for (int l = 0; l < 4; l++) e1[l] = (t[l] >> 2) | (l < 3 ? t[l + 1] << 62 : 0);
        for (int l = 0; l < 4; l++) e2[l] = (FQ_P.p[l] >> 1) | (l < 3 ? FQ_P.p[l + 1] << 63 : 0);   // (q - 1) / 2
    }
    const Fq2 a1 = pw(a, e1);
    const Fq2 x0 = a1 * a;
    const Fq2 alpha = a1 * x0;
    Fq2 minus_one = {-Fq::one(), Fq::zero()};
    Fq2 x;
    if (alpha == minus_one) {
        x = {-x0.c1, x0.c0};   // u x0
    } else {
        const Fq2 b = pw(alpha + Fq2::one(), e2);
        x = b * x0;
    }
    out = x;
    return x.sqr() == a;
}

bool encoder_g1(Reader& r, G1A& p) {
    const uint8_t* b = r.take(32);
    if (!b) return false;
    const int flag = b[0] >> 6;
    uint8_t x[32];
    std::memcpy(x, b, 32);
    x[0] &= 0x3f;
    p.inf = false;
    if (flag == 1) {
        p.inf = true;
        p.x = p.y = Fq::zero();
        return true;
    }
    if (!be_elem(x, p.x)) return r.fail("G1 x is not below q");
    if (flag == 0) {
        const uint8_t* yb = r.take(32);
        if (!yb) return false;
        static const uint8_t zero[32] = {};
        if (!std::memcmp(x, zero, 32) && !std::memcmp(yb, zero, 32)) {
            p.inf = true;
            p.x = p.y = Fq::zero();
            return true;
        }
        if (!be_elem(yb, p.y)) return r.fail("G1 y is not below q");
    } else {
        if (!fq_sqrt(p.x.sqr() * p.x + Fq::from_u64(3), p.y)) return r.fail("compressed G1 x is not on the curve");
        if (fq_larger(p.y) != (flag == 3)) p.y = -p.y;
    }
    if (!on_curve(p)) return r.fail("G1 point is not on the curve");
    return true;
}

bool encoder_g2(Reader& r, G2A& p) {
    const uint8_t* b = r.take(64);
    if (!b) return false;
    const int flag = b[0] >> 6;
    uint8_t x1[32];
    std::memcpy(x1, b, 32);
    x1[0] &= 0x3f;
    p.inf = false;
    if (flag == 1) {
        p.inf = true;
        p.x = p.y = Fq2::zero();
        return true;
    }
    if (!be_elem(x1, p.x.c1) || !be_elem(b + 32, p.x.c0)) return r.fail("G2 x is not below q");
    if (flag == 0) {
        const uint8_t* yb = r.take(64);
        if (!yb) return false;
        static const uint8_t zero[64] = {};
        if (!std::memcmp(b, zero, 64) && !std::memcmp(yb, zero, 64)) {
            p.inf = true;
            p.x = p.y = Fq2::zero();
            return true;
        }
        if (!be_elem(yb, p.y.c1) || !be_elem(yb + 32, p.y.c0)) return r.fail("G2 y is not below q");
    } else {
        if (!fq2_sqrt(p.x.sqr() * p.x + TWIST_B, p.y)) return r.fail("compressed G2 x is not on the curve");
        const bool larger = p.y.c1.is_zero() ? fq_larger(p.y.c0) : fq_larger(p.y.c1);
        if (larger != (flag == 3)) p.y = -p.y;
    }
    if (!on_curve(p)) return r.fail("G2 point is not on the curve");
    return true;
}

bool same(const G1A& a, const G1A& b) { return a.inf == b.inf && (a.inf || (a.x == b.x && a.y == b.y)); }
bool same(const G2A& a, const G2A& b) { return a.inf == b.inf && (a.inf || (a.x == b.x && a.y == b.y)); }

template <class P>
std::vector<uint8_t> packed(const P& p, size_t bytes) {
    std::vector<uint8_t> v(bytes);
    pack(v.data(), p);
    return v;
}

// dumped query points: canonical coordinates on the curve (infinity = zeros)
template <class P>
bool check_points(Reader& r, const uint8_t* d, size_t n, size_t stride) {
    for (size_t i = 0; i < n; i++) {
        P p;
        if (!unpack(p, d + i * stride)) return r.fail("a dumped point has a coordinate not below q");
        if (!on_curve(p)) return r.fail("a dumped point is not on the curve");
    }
    return true;
}

}  // namespace

int gnark_key_parse(const uint8_t* pk, size_t pk_len, const uint8_t* vk, size_t vk_len, ZkeyHost& k) {
    host_init();
    k = ZkeyHost();
    Reader r{pk, pk_len};
    r.part = "dump marker";
    static const uint8_t marker[8] = {0xef, 0xbe, 0xad, 0xde, 0, 0, 0, 0};
    const uint8_t* m = r.take(8);
    if (!m || std::memcmp(m, marker, 8)) {
        if (r.ok) r.fail("not a little-endian gnark dump");
        return G16_ERR_FORMAT;
    }
    // Domain.WriteTo: cardinality, 1/n, generator, its inverse, the multiplicative generator and its inverse
    r.part = "domain";
    uint64_t card = 0;
    if (!r.be(8, card)) return G16_ERR_FORMAT;
    if (card < 2 || (card & (card - 1)) || card > (1ull << 27)) {
        r.fail("cardinality is not a power of two in [2, 2^27]");
        return G16_ERR_FORMAT;
    }
    int log_n = 0;
    while ((1ull << log_n) < card) log_n++;
    Fr dom[5];
    for (auto& e : dom) {
        const uint8_t* b = r.take(32);
        if (!b) return G16_ERR_FORMAT;
        if (!be_elem(b, e)) {
            r.fail("a domain scalar is not below r");
            return G16_ERR_FORMAT;
        }
    }
    // the library squares the same 2^28-th root of unity down: another generator
    // would make the prover's H not pair with this key's Z
    if (!(dom[0] == Fr::from_u64(card).inv()) || !(dom[1] == domain_root(log_n))) {
        r.fail("the domain is not the one this prover uses for its size");
        return G16_ERR_FORMAT;
    }
    const uint8_t* pre = r.take(1);
    if (!pre || *pre > 1) {
        if (r.ok) r.fail("precompute byte is not a bool");
        return G16_ERR_FORMAT;
    }
    r.part = "header points";
    G1A alpha, beta1, delta1;
    G2A beta2, delta2;
    if (!encoder_g1(r, alpha) || !encoder_g1(r, beta1) || !encoder_g1(r, delta1) || !encoder_g2(r, beta2) ||
        !encoder_g2(r, delta2))
        return G16_ERR_FORMAT;
    if (alpha.inf || beta1.inf || delta1.inf || beta2.inf || delta2.inf) {
        r.fail("a header point is the point at infinity");
        return G16_ERR_FORMAT;
    }
    r.part = "wire counts";
    uint64_t nw = 0, ninf_a = 0, ninf_b = 0;
    if (!r.be(8, nw) || !r.be(8, ninf_a) || !r.be(8, ninf_b)) return G16_ERR_FORMAT;
    if (nw < 1 || nw > pk_len || nw >= 0x80000000ull) {
        r.fail("wire count out of range");
        return G16_ERR_FORMAT;
    }
    r.part = "infinity flags";
    const uint8_t* fa = r.take(nw);
    const uint8_t* fb = r.take(nw);
    if (!fa || !fb) return G16_ERR_FORMAT;
    uint64_t ca = 0, cb = 0;
    for (uint64_t i = 0; i < nw; i++) {
        if (fa[i] > 1 || fb[i] > 1) {
            r.fail("a flag is not a bool");
            return G16_ERR_FORMAT;
        }
        ca += fa[i];
        cb += fb[i];
    }
    if (ca != ninf_a || cb != ninf_b) {
        r.fail("the set flags do not match the header's counts");
        return G16_ERR_FORMAT;
    }
    r.part = "commitments";
    uint64_t ncommit = 0;
    if (!r.be(4, ncommit)) return G16_ERR_FORMAT;
    if (ncommit) {
        r.fail("BSB22 commitment keys are not supported");
        return G16_ERR_FORMAT;
    }
    size_t na = 0, nb = 0, nz = 0, nk = 0, nb2 = 0;
    r.part = "G1.A";
    const uint8_t* sa = r.dumped(64, na);
    r.part = "G1.B";
    const uint8_t* sb = r.dumped(64, nb);
    r.part = "G1.Z";
    const uint8_t* sz = r.dumped(64, nz);
    r.part = "G1.K";
    const uint8_t* sk = r.dumped(64, nk);
    r.part = "G2.B";
    const uint8_t* sb2 = r.dumped(128, nb2);
    if (!r.ok) return G16_ERR_FORMAT;
    r.part = "trailer";
    if (r.pos != r.len) {
        r.fail("trailing bytes");
        return G16_ERR_FORMAT;
    }
    r.part = "slice lengths";
    if (na != nw - ca || nb != nw - cb || nb2 != nw - cb || nz != card - 1 || nk >= nw) {
        r.fail("a dumped query's length does not match the header");
        return G16_ERR_FORMAT;
    }
    r.part = "query points";
    if (!check_points<G1A>(r, sa, na, 64) || !check_points<G1A>(r, sb, nb, 64) || !check_points<G1A>(r, sz, nz, 64) ||
        !check_points<G1A>(r, sk, nk, 64) || !check_points<G2A>(r, sb2, nb2, 128))
        return G16_ERR_FORMAT;

    // the verifying key: gamma and the public wires' K (the IC)
    Reader v{vk, vk_len};
    v.part = "verifying key";
    G1A valpha, vbeta1, vdelta1;
    G2A vbeta2, vgamma2, vdelta2;
    if (!encoder_g1(v, valpha) || !encoder_g1(v, vbeta1) || !encoder_g2(v, vbeta2) || !encoder_g2(v, vgamma2) ||
        !encoder_g1(v, vdelta1) || !encoder_g2(v, vdelta2))
        return G16_ERR_FORMAT;
    if (!same(valpha, alpha) || !same(vbeta1, beta1) || !same(vdelta1, delta1) || !same(vbeta2, beta2) ||
        !same(vdelta2, delta2)) {
        v.fail("its alpha, beta or delta differs from the proving key's");
        return G16_ERR_FORMAT;
    }
    if (vgamma2.inf) {
        v.fail("gamma is the point at infinity");
        return G16_ERR_FORMAT;
    }
    uint64_t nic = 0;
    if (!v.be(4, nic)) return G16_ERR_FORMAT;
    if (nic != nw - nk || nic < 1) {
        v.fail("its K points do not match the proving key's public wires");
        return G16_ERR_FORMAT;
    }
    std::vector<G1A> ic(nic);
    for (auto& p : ic)
        if (!encoder_g1(v, p)) return G16_ERR_FORMAT;
    uint64_t committed = 0, commitments = 0;
    if (!v.be(4, committed) || !v.be(4, commitments)) return G16_ERR_FORMAT;
    if (committed || commitments) {
        v.fail("BSB22 commitments are not supported");
        return G16_ERR_FORMAT;
    }
    if (v.pos != v.len) {
        v.fail("trailing bytes");
        return G16_ERR_FORMAT;
    }

    k.n_vars = (uint32_t)nw;
    k.n_public = (uint32_t)nic - 1;
    k.domain_size = (uint32_t)card;
    k.h_basis = 1;
    k.alpha_g1 = packed(alpha, 64);
    k.beta_g1 = packed(beta1, 64);
    k.delta_g1 = packed(delta1, 64);
    k.beta_g2 = packed(beta2, 128);
    k.gamma_g2 = packed(vgamma2, 128);
    k.delta_g2 = packed(delta2, 128);
    k.ic.resize(64 * nic);
    for (size_t i = 0; i < nic; i++) pack(k.ic.data() + 64 * i, ic[i]);
    // one base per wire: the flagged wires are the point at infinity (zeros)
    k.a_query.assign(64 * nw, 0);
    k.b_g1_query.assign(64 * nw, 0);
    k.b_g2_query.assign(128 * nw, 0);
    size_t ia = 0, ib = 0;
    for (uint64_t i = 0; i < nw; i++) {
        if (!fa[i]) std::memcpy(&k.a_query[64 * i], sa + 64 * ia++, 64);
        if (!fb[i]) {
            std::memcpy(&k.b_g1_query[64 * i], sb + 64 * ib, 64);
            std::memcpy(&k.b_g2_query[128 * i], sb2 + 128 * ib, 128);
            ib++;
        }
    }
    k.l_query.assign(sk, sk + 64 * nk);
    k.h_query.assign(sz, sz + 64 * nz);
    return G16_OK;
}

int gnark_witness_parse(const uint8_t* d, size_t len, std::vector<uint8_t> out[3]) {
    host_init();
    Reader r{d, len};
    r.part = "witness";
    static const uint8_t marker[8] = {0xef, 0xbe, 0xad, 0xde, 0, 0, 0, 0};
    const uint8_t* m = r.take(8);
    if (!m || std::memcmp(m, marker, 8)) {
        if (r.ok) r.fail("not a little-endian gnark dump");
        return G16_ERR_FORMAT;
    }
    const char* names[3] = {"W", "Aw", "Bw"};
    for (int s = 0; s < 3; s++) {
        r.part = names[s];
        size_t n = 0;
        const uint8_t* p = r.dumped(32, n);
        if (!p) return G16_ERR_FORMAT;
        for (size_t i = 0; i < n; i++) {
            uint64_t v[4];
            std::memcpy(v, p + 32 * i, 32);
            if (!Fr::canonical(v)) {
                r.fail("an element is not below r");
                return G16_ERR_FORMAT;
            }
        }
        out[s].assign(p, p + 32 * n);
    }
    r.part = "trailer";
    if (r.pos != r.len) {
        r.fail("trailing bytes");
        return G16_ERR_FORMAT;
    }
    if (out[1].size() != out[2].size()) {
        set_error("gnark witness: A.w and B.w have different lengths");
        return G16_ERR_FORMAT;
    }
    const Fr one = Fr::one();
    if (out[0].size() < 32 || std::memcmp(out[0].data(), one.x.v, 32) != 0) {
        set_error("gnark witness: W[0] is not 1");
        return G16_ERR_FORMAT;
    }
    return G16_OK;
}

}  // namespace g16
