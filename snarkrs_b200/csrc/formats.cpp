// snarkjs .zkey / .wtns readers and writers (the input boundary of the
// prover), restating crates/formats/src/lib.rs and binfile.rs:
//   iden3 binfile container (binfile.rs:10-26): 4-byte magic, u32 version,
//   u32 nSections, then (u32 id, u64 length, payload) in any order, ids
//   unique for the sections read;
//   zkey sections 1-10 (lib.rs:1-16); points are Montgomery limbs verbatim
//   with (0,0) = infinity and limbs >= q refused (binfile.rs:465-540);
//   section 4 values are double Montgomery v*R^2, decoded with one
//   Montgomery multiply by the raw integer 1 (binfile.rs:505-520);
//   section 4 sorted by (matrix, constraint) into CSR with interned values
//   (lib.rs:140-223, read_coefficients :905);
//   .wtns values plain little-endian integers, w[0] must be 1 (wtns.rs:17-40).
#include "formats.hpp"
#include "common.cuh"
#include "g16b200.h"
#include <unordered_map>

namespace g16 {

static uint32_t rd32(const uint8_t* b) { uint32_t x; std::memcpy(&x, b, 4); return x; }
static uint64_t rd64(const uint8_t* b) { uint64_t x; std::memcpy(&x, b, 8); return x; }

struct Sec {
    uint32_t id;
    size_t off, len;
};

static bool scan_sections(const uint8_t* d, size_t len, const char* magic, std::vector<Sec>& out) {
    if (len < 12 || std::memcmp(d, magic, 4) != 0) {
        set_error("not a %s file (magic)", magic);
        return false;
    }
    uint32_t ns = rd32(d + 8);
    size_t off = 12;
    for (uint32_t i = 0; i < ns; i++) {
        if (off + 12 > len) {
            set_error("%s: truncated section header %u", magic, i);
            return false;
        }
        Sec s;
        s.id = rd32(d + off);
        uint64_t l = rd64(d + off + 4);
        s.off = off + 12;
        if (l > len - s.off) {
            set_error("%s: section %u declares %llu bytes past the end", magic, s.id, (unsigned long long)l);
            return false;
        }
        s.len = (size_t)l;
        off = s.off + s.len;
        out.push_back(s);
    }
    return true;
}

static const Sec* unique(const std::vector<Sec>& v, uint32_t id) {
    const Sec* hit = nullptr;
    for (auto& s : v)
        if (s.id == id) {
            if (hit) {
                set_error("section %u appears twice", id);
                return nullptr;
            }
            hit = &s;
        }
    if (!hit) set_error("section %u is missing", id);
    return hit;
}

static bool canonical_points(const uint8_t* p, size_t n, size_t stride, bool check_curve, uint32_t section) {
    for (size_t i = 0; i < n; i++) {
        const uint8_t* q = p + i * stride;
        if (stride == 64) {
            G1A a;
            if (!unpack(a, q)) {
                set_error("section %u point %zu: coordinate not below q", section, i);
                return false;
            }
            if (check_curve && !on_curve(a)) {
                set_error("section %u point %zu is not on the curve", section, i);
                return false;
            }
        } else {
            G2A a;
            if (!unpack(a, q)) {
                set_error("section %u point %zu: coordinate not below q", section, i);
                return false;
            }
            if (check_curve && !on_curve(a)) {
                set_error("section %u point %zu is not on the curve", section, i);
                return false;
            }
        }
    }
    return true;
}

int zkey_parse(const uint8_t* d, size_t len, bool check_points, ZkeyHost& k) {
    host_init();
    std::vector<Sec> secs;
    if (!scan_sections(d, len, "zkey", secs)) return G16_ERR_FORMAT;
    const Sec* s1 = unique(secs, 1);
    const Sec* s2 = unique(secs, 2);
    if (!s1 || !s2) return G16_ERR_FORMAT;
    if (s1->len < 4 || rd32(d + s1->off) != 1) {
        set_error("zkey protocol is not groth16");
        return G16_ERR_FORMAT;
    }
    const uint8_t* h = d + s2->off;
    if (s2->len != 84 + 64 * 3 + 128 * 3) {
        set_error("zkey section 2 has %zu bytes, expected 660", s2->len);
        return G16_ERR_FORMAT;
    }
    if (rd32(h) != 32 || std::memcmp(h + 4, FQ_P.p, 32) != 0 || rd32(h + 36) != 32 ||
        std::memcmp(h + 40, FR_P.p, 32) != 0) {
        set_error("zkey is not over BN254");
        return G16_ERR_FORMAT;
    }
    k.n_vars = rd32(h + 72);
    k.n_public = rd32(h + 76);
    k.domain_size = rd32(h + 80);
    uint32_t n = k.domain_size;
    if (n == 0 || (n & (n - 1)) || n > (1u << 27)) {
        set_error("zkey domain size %u is not a power of two in [1, 2^27]", n);
        return G16_ERR_FORMAT;
    }
    if ((uint64_t)k.n_public + 1 > k.n_vars) {
        set_error("n_vars %u does not cover 1 + n_public %u", k.n_vars, k.n_public);
        return G16_ERR_FORMAT;
    }
    const uint8_t* pt = h + 84;
    k.alpha_g1.assign(pt, pt + 64);
    k.beta_g1.assign(pt + 64, pt + 128);
    k.beta_g2.assign(pt + 128, pt + 256);
    k.gamma_g2.assign(pt + 256, pt + 384);
    k.delta_g1.assign(pt + 384, pt + 448);
    k.delta_g2.assign(pt + 448, pt + 576);
    {
        G1A a;
        G2A b;
        const uint8_t* g1s[3] = {k.alpha_g1.data(), k.beta_g1.data(), k.delta_g1.data()};
        const uint8_t* g2s[3] = {k.beta_g2.data(), k.gamma_g2.data(), k.delta_g2.data()};
        for (auto p : g1s)
            if (!unpack(a, p) || a.inf || !on_curve(a)) {
                set_error("zkey header G1 point is invalid or the point at infinity");
                return G16_ERR_FORMAT;
            }
        for (auto p : g2s)
            if (!unpack(b, p) || b.inf || !on_curve(b)) {
                set_error("zkey header G2 point is invalid or the point at infinity");
                return G16_ERR_FORMAT;
            }
    }
    const Sec* s[11] = {};
    for (uint32_t id = 3; id <= 9; id++)
        if (!(s[id] = unique(secs, id))) return G16_ERR_FORMAT;
    size_t nv = k.n_vars, nic = (size_t)k.n_public + 1, nl = nv - nic;
    struct Want {
        uint32_t id;
        size_t n, stride;
    } want[] = {{3, nic, 64}, {5, nv, 64}, {6, nv, 64}, {7, nv, 128}, {8, nl, 64}, {9, n, 64}};
    for (auto& w : want) {
        if (s[w.id]->len != w.n * w.stride) {
            set_error("zkey section %u: expected %zu records of %zu bytes, got %zu bytes", w.id, w.n, w.stride,
                      s[w.id]->len);
            return G16_ERR_FORMAT;
        }
        if (!canonical_points(d + s[w.id]->off, w.n, w.stride, check_points || w.id == 3, w.id))
            return G16_ERR_FORMAT;
    }
    k.ic.assign(d + s[3]->off, d + s[3]->off + s[3]->len);
    k.a_query.assign(d + s[5]->off, d + s[5]->off + s[5]->len);
    k.b_g1_query.assign(d + s[6]->off, d + s[6]->off + s[6]->len);
    k.b_g2_query.assign(d + s[7]->off, d + s[7]->off + s[7]->len);
    k.l_query.assign(d + s[8]->off, d + s[8]->off + s[8]->len);
    k.h_query.assign(d + s[9]->off, d + s[9]->off + s[9]->len);

    // section 4 -> CSR
    const uint8_t* c4 = d + s[4]->off;
    if (s[4]->len < 4) {
        set_error("zkey section 4 is too short");
        return G16_ERR_FORMAT;
    }
    uint32_t ncoef = rd32(c4);
    if ((size_t)ncoef * 44 != s[4]->len - 4) {
        set_error("zkey section 4: %u records do not fill %zu bytes", ncoef, s[4]->len - 4);
        return G16_ERR_FORMAT;
    }
    for (int m = 0; m < 2; m++) k.row_ptr[m].assign((size_t)n + 1, 0);
    for (uint32_t i = 0; i < ncoef; i++) {
        const uint8_t* r = c4 + 4 + 44 * (size_t)i;
        uint32_t m = rd32(r), c = rd32(r + 4), sg = rd32(r + 8);
        if (m > 1) {
            set_error("zkey section 4 record %u: matrix %u", i, m);
            return G16_ERR_FORMAT;
        }
        if (c >= n) {
            set_error("zkey section 4 record %u: constraint %u is outside domain size %u", i, c, n);
            return G16_ERR_FORMAT;
        }
        if (sg >= k.n_vars) {
            set_error("zkey section 4 record %u: signal %u beyond n_vars %u", i, sg, k.n_vars);
            return G16_ERR_FORMAT;
        }
        k.row_ptr[m][c + 1]++;
    }
    for (int m = 0; m < 2; m++) {
        for (uint32_t c = 0; c < n; c++) k.row_ptr[m][c + 1] += k.row_ptr[m][c];
        size_t nnz = k.row_ptr[m][n];
        k.signal[m].assign(nnz, 0);
        k.value_id[m].assign(nnz, 0);
    }
    std::vector<uint32_t> cur[2] = {k.row_ptr[0], k.row_ptr[1]};
    struct H32 {
        size_t operator()(const Fe& x) const { return (size_t)(x.v[0] ^ (x.v[1] * 0x9E3779B97F4A7C15ULL) ^ x.v[2] ^ x.v[3]); }
    };
    struct E32 {
        bool operator()(const Fe& a, const Fe& b) const { return std::memcmp(a.v, b.v, 32) == 0; }
    };
    std::unordered_map<Fe, uint32_t, H32, E32> ids;
    ids.reserve(1024);
    k.values.clear();
    Fr one_raw = Fr::zero();
    one_raw.x.v[0] = 1;
    for (uint32_t i = 0; i < ncoef; i++) {
        const uint8_t* r = c4 + 4 + 44 * (size_t)i;
        uint32_t m = rd32(r), c = rd32(r + 4), sg = rd32(r + 8);
        uint64_t raw[4];
        std::memcpy(raw, r + 12, 32);
        if (!Fr::canonical(raw)) {
            set_error("zkey section 4 record %u: value not below r", i);
            return G16_ERR_FORMAT;
        }
        Fr v = Fr::raw(raw) * one_raw;   // v R^2 -> v R
        auto it = ids.find(v.x);
        uint32_t id;
        if (it == ids.end()) {
            id = (uint32_t)(k.values.size() / 32);
            ids.emplace(v.x, id);
            k.values.insert(k.values.end(), (const uint8_t*)v.x.v, (const uint8_t*)v.x.v + 32);
        } else {
            id = it->second;
        }
        uint32_t at = cur[m][c]++;
        k.signal[m][at] = sg;
        k.value_id[m][at] = id;
    }
    return G16_OK;
}

void zkey_view(const ZkeyHost& k, g16_zkey_view& v) {
    v.n_vars = k.n_vars;
    v.n_public = k.n_public;
    v.domain_size = k.domain_size;
    v.alpha_g1 = k.alpha_g1.data();
    v.beta_g1 = k.beta_g1.data();
    v.beta_g2 = k.beta_g2.data();
    v.gamma_g2 = k.gamma_g2.data();
    v.delta_g1 = k.delta_g1.data();
    v.delta_g2 = k.delta_g2.data();
    v.ic = k.ic.data();
    for (int m = 0; m < 2; m++) {
        v.row_ptr[m] = k.row_ptr[m].data();
        v.signal[m] = k.signal[m].data();
        v.value_id[m] = k.value_id[m].data();
        v.nnz[m] = (uint32_t)k.signal[m].size();
    }
    v.values = k.values.data();
    v.n_values = (uint32_t)(k.values.size() / 32);
    v.a_query = k.a_query.data();
    v.b_g1_query = k.b_g1_query.data();
    v.b_g2_query = k.b_g2_query.data();
    v.l_query = k.l_query.data();
    v.h_query = k.h_query.data();
    v.h_basis = k.h_basis;
}

int wtns_parse(const uint8_t* d, size_t len, std::vector<uint8_t>& out_mont) {
    host_init();
    std::vector<Sec> secs;
    if (!scan_sections(d, len, "wtns", secs)) return G16_ERR_FORMAT;
    const Sec* s1 = unique(secs, 1);
    const Sec* s2 = unique(secs, 2);
    if (!s1 || !s2) return G16_ERR_FORMAT;
    if (s1->len < 40 || rd32(d + s1->off) != 32 || std::memcmp(d + s1->off + 4, FR_P.p, 32) != 0) {
        set_error("wtns is not over the BN254 scalar field");
        return G16_ERR_FORMAT;
    }
    uint32_t nw = rd32(d + s1->off + 36);
    if ((size_t)nw * 32 != s2->len) {
        set_error("wtns section 2 holds %zu bytes for %u values", s2->len, nw);
        return G16_ERR_FORMAT;
    }
    out_mont.resize((size_t)nw * 32);
    for (uint32_t i = 0; i < nw; i++) {
        uint64_t raw[4];
        std::memcpy(raw, d + s2->off + 32 * (size_t)i, 32);
        if (!Fr::canonical(raw)) {
            set_error("wtns value %u is not below the scalar modulus", i);
            return G16_ERR_FORMAT;
        }
        Fr v = Fr::from_std(raw);
        std::memcpy(out_mont.data() + 32 * (size_t)i, v.x.v, 32);
    }
    if (nw == 0 || !(Fr::raw((const uint64_t*)out_mont.data()) == Fr::one())) {
        set_error("witness[0] is not 1");
        return G16_ERR_FORMAT;
    }
    return G16_OK;
}

void BinWriter::begin(const char* magic, uint32_t version, uint32_t nsec) {
    buf.insert(buf.end(), magic, magic + 4);
    u32(version);
    u32(nsec);
}
void BinWriter::section(uint32_t id) {
    u32(id);
    sec_start = buf.size();
    u64(0);
}
void BinWriter::end_section() {
    uint64_t l = buf.size() - sec_start - 8;
    std::memcpy(buf.data() + sec_start, &l, 8);
}

std::vector<uint8_t> wtns_write(const uint8_t* w_mont, size_t n) {
    host_init();
    BinWriter w;
    w.begin("wtns", 2, 2);
    w.section(1);
    w.u32(32);
    w.bytes(FR_P.p, 32);
    w.u32((uint32_t)n);
    w.end_section();
    w.section(2);
    for (size_t i = 0; i < n; i++) {
        uint64_t v[4], s[4];
        std::memcpy(v, w_mont + 32 * i, 32);
        Fr::raw(v).to_std(s);
        w.bytes(s, 32);
    }
    w.end_section();
    return std::move(w.buf);
}

}  // namespace g16
