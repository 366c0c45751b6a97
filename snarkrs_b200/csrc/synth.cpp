// Seeded synthetic circuits, witnesses and proving keys.
//
// The circuit: wire 0 = 1, n_inputs input wires (the first n_public public),
// and per constraint one new wire w_k := (A.w)(B.w) with 2-3 terms in each of
// A and B on wires defined earlier, so every witness satisfies it by
// construction.  Each constraint is given a value class up front -- 0 or 1
// (60%), below 2^32 (20%), uniform (20%) -- and its rows are shaped so the
// product lands in that class for every choice of inputs: a 1 is (1*one +
// zeros)(1*one + zeros), a 0 is (one - one')(anything), a small value is a
// 16-bit coefficient on a one-wire or a product of two 16-bit wires, a
// uniform value multiplies rows led by a uniform wire with a uniform
// coefficient.  Extra terms sit on zero wires with coefficients uniform in Fr
// or +-1, so they change no value.  The first constraints have fewer terms
// while the pools of zero and one wires fill.
//
// The key: a snarkjs Groth16 .zkey written directly from seeded toxic waste
// (tau, alpha, beta, delta; gamma = 1), with the semantics of snarkjs'
// zkey_new + zkey_contribute as the reference restates them
// (crates/ceremony/src/setup.rs:1-30, 133-170, 760-1000 and contribute.rs):
//   domain = 2^(floor(log2(nConstraints + nPublic)) + 1);
//   one extra A row per public signal s (row nConstraints + s, coefficient 1);
//   A_j = [u_j(tau)]_1, B1_j = [v_j(tau)]_1, B2_j = [v_j(tau)]_2 with u, v, w
//   the columns of A, B, C in the Lagrange basis of the domain;
//   IC_j = [beta u_j + alpha v_j + w_j]_1 for j <= nPublic (gamma = 1);
//   L_j  = [(beta u_j + alpha v_j + w_j) / delta]_1 for the private wires;
//   H_i  = [L^(2n)_(2i+1)(tau) / delta]_1, the odd Lagrange basis of the 2n
//          domain (setup.rs:16-20, zkey_new writeHs);
//   section 4 = the A and B coefficients as double-Montgomery records;
//   sections written in snarkjs order 1, 2, 4, 3, 9, 8, 5, 6, 7, 10.
#include "common.cuh"
#include "formats.hpp"
#include "g16b200.h"
#include "host_bn254.hpp"
#include "msm.cuh"
#include <algorithm>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>

using namespace g16;

namespace {

struct SplitMix {
    uint64_t s;
    uint64_t next() {
        s += 0x9E3779B97F4A7C15ULL;
        uint64_t z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    uint32_t below(uint32_t n) { return (uint32_t)(((unsigned __int128)next() * n) >> 64); }
    // uniform in [0, r): 254 random bits, one conditional subtraction
    Fr fr() {
        uint64_t v[4] = {next(), next(), next(), next() & ((1ULL << 62) - 1)};
        if (geq4(v, FR_P.p)) sub4(v, v, FR_P.p);
        return Fr::from_std(v);
    }
    Fr fr_nonzero() {
        for (;;) {
            Fr x = fr();
            if (!x.is_zero()) return x;
        }
    }
};

enum Cls : uint8_t { ZERO = 0, ONE = 1, SMALL16 = 2, SMALL32 = 3, UNIF = 4 };

struct Term {
    uint32_t sig;
    Fr coef;
};

}  // namespace

struct g16_synth {
    uint32_t n_constraints, n_inputs, n_public, n_vars, domain;
    // rows of A and B, CSR by constraint; C row k is 1 * w[1 + n_inputs + k]
    std::vector<uint32_t> ptr[2];
    std::vector<Term> terms[2];
    std::mutex mu;
    uint64_t cached_seed = 0;
    bool cached = false;
    std::vector<uint8_t> zkey;
};

static void build_structure(g16_synth& s, uint64_t seed) {
    SplitMix rng{seed};
    std::vector<uint32_t> pool[5];
    pool[ONE].push_back(0);
    for (uint32_t i = 1; i <= s.n_inputs; i++) pool[UNIF].push_back(i);
    const Fr one = Fr::one(), minus_one = -Fr::one();
    auto coef = [&]() { return (rng.next() & 1) ? rng.fr() : ((rng.next() & 1) ? one : minus_one); };
    auto pick = [&](int c) { return pool[c][rng.below((uint32_t)pool[c].size())]; };
    for (int m = 0; m < 2; m++) {
        s.ptr[m].assign(1, 0);
        s.terms[m].reserve((size_t)s.n_constraints * 5 / 2);
    }
    for (uint32_t k = 0; k < s.n_constraints; k++) {
        uint32_t out = 1 + s.n_inputs + k;
        double r = rng.uniform();
        int cls = r < 0.30 ? ZERO : r < 0.60 ? ONE : r < 0.70 ? SMALL16 : r < 0.80 ? SMALL32 : UNIF;
        if (cls == ZERO && pool[ONE].size() < 2) cls = ONE;
        if (cls == SMALL32 && pool[SMALL16].empty()) cls = SMALL16;
        uint32_t na = 2 + (uint32_t)(rng.next() & 1), nb = 2 + (uint32_t)(rng.next() & 1);
        std::vector<Term> a, b;
        auto zeros = [&](std::vector<Term>& row, uint32_t want) {
            while (row.size() < want && !pool[ZERO].empty()) row.push_back({pick(ZERO), coef()});
        };
        auto anywire = [&](std::vector<Term>& row, uint32_t want) {
            while (row.size() < want) row.push_back({rng.below(out), coef()});
        };
        switch (cls) {
            case ONE:
                a.push_back({pick(ONE), one});
                b.push_back({pick(ONE), one});
                zeros(a, na);
                zeros(b, nb);
                break;
            case ZERO: {
                uint32_t o1 = pick(ONE), o2;
                do o2 = pick(ONE);
                while (o2 == o1);
                a.push_back({o1, one});
                a.push_back({o2, minus_one});
                zeros(a, na);
                anywire(b, nb);
                break;
            }
            case SMALL16: {
                uint64_t v = 2 + rng.below((1u << 16) - 2);
                a.push_back({pick(ONE), Fr::from_u64(v)});
                b.push_back({pick(ONE), one});
                zeros(a, na);
                zeros(b, nb);
                break;
            }
            case SMALL32:
                a.push_back({pick(SMALL16), one});
                b.push_back({pick(SMALL16), one});
                zeros(a, na);
                zeros(b, nb);
                break;
            default:
                a.push_back({pick(UNIF), rng.fr_nonzero()});
                b.push_back({pick(UNIF), rng.fr_nonzero()});
                anywire(a, na);
                anywire(b, nb);
                break;
        }
        pool[cls].push_back(out);
        s.terms[0].insert(s.terms[0].end(), a.begin(), a.end());
        s.terms[1].insert(s.terms[1].end(), b.begin(), b.end());
        s.ptr[0].push_back((uint32_t)s.terms[0].size());
        s.ptr[1].push_back((uint32_t)s.terms[1].size());
    }
}

static void compute_witness(const g16_synth& s, uint64_t wseed, std::vector<Fr>& w) {
    SplitMix rng{wseed ^ 0x5bd1e995a3c5f7e1ULL};
    w.assign(s.n_vars, Fr::zero());
    w[0] = Fr::one();
    for (uint32_t i = 1; i <= s.n_inputs; i++) w[i] = rng.fr();
    for (uint32_t k = 0; k < s.n_constraints; k++) {
        Fr av = Fr::zero(), bv = Fr::zero();
        for (uint32_t t = s.ptr[0][k]; t < s.ptr[0][k + 1]; t++) av = av + s.terms[0][t].coef * w[s.terms[0][t].sig];
        for (uint32_t t = s.ptr[1][k]; t < s.ptr[1][k + 1]; t++) bv = bv + s.terms[1][t].coef * w[s.terms[1][t].sig];
        w[1 + s.n_inputs + k] = av * bv;
    }
}

// fixed-base scalar multiplication with 8-bit windows: table[w][d] = d 2^(8w) G
template <class F>
struct FixedBase {
    std::vector<Affine<F>> t;
    explicit FixedBase(const Affine<F>& g) {
        std::vector<Jac<F>> j(32 * 256);
        Jac<F> base = Jac<F>::from_affine(g);
        for (int w = 0; w < 32; w++) {
            Jac<F> cur = Jac<F>::identity();
            for (int d = 0; d < 256; d++) {
                j[w * 256 + d] = cur;
                cur = cur + base;
            }
            for (int k = 0; k < 8; k++) base = base.dbl();
        }
        t.resize(j.size());
        batch_to_affine(j.data(), t.data(), j.size());
    }
    Jac<F> mul(const Fr& k) const {
        uint64_t s[4];
        k.to_std(s);
        Jac<F> acc = Jac<F>::identity();
        for (int w = 0; w < 32; w++) {
            unsigned d = (unsigned)((s[w / 8] >> (8 * (w % 8))) & 255);
            if (d) acc = acc.add_affine(t[w * 256 + d]);
        }
        return acc;
    }
};

template <class F>
static void points_into(const FixedBase<F>& fb, const Fr* scalars, size_t n, uint8_t* out, size_t stride,
                        int threads) {
    auto work = [&](size_t lo, size_t hi) {
        const size_t CH = 4096;
        std::vector<Jac<F>> j(CH);
        std::vector<Affine<F>> a(CH);
        for (size_t c0 = lo; c0 < hi; c0 += CH) {
            size_t c1 = std::min(hi, c0 + CH);
            for (size_t i = c0; i < c1; i++) j[i - c0] = fb.mul(scalars[i]);
            batch_to_affine(j.data(), a.data(), c1 - c0);
            for (size_t i = c0; i < c1; i++) pack(out + i * stride, a[i - c0]);
        }
    };
    std::vector<std::thread> pool;
    size_t per = (n + threads - 1) / threads;
    for (int t = 0; t < threads; t++) {
        size_t lo = t * per, hi = std::min(n, lo + per);
        if (lo >= hi) break;
        pool.emplace_back(work, lo, hi);
    }
    for (auto& th : pool) th.join();
}

// Where the key's point sections are computed: out[i * stride] = k_i G for the
// group's generator (1 = G1, 2 = G2), packed affine.  Returns false on failure
// (error set).
typedef std::function<bool(int group, const Fr* scalars, size_t n, uint8_t* out)> PointsFn;

// The device path: the same fixed-base 8-bit-window sums on the GPU
// (fixed_base_g1/g2), normalised with batched inversions, bit-identical.
struct DevicePoints {
    int device;
    cudaStream_t st = nullptr;
    void *d_t1 = nullptr, *d_t2 = nullptr, *d_k = nullptr, *d_out = nullptr;
    size_t cap_k = 0, cap_out = 0;
    bool ok = true;
    explicit DevicePoints(int dev) : device(dev) {}
    ~DevicePoints() {
        for (void* p : {d_t1, d_t2, d_k, d_out})
            if (p) cudaFree(p);
        if (st) cudaStreamDestroy(st);
    }
    bool check(cudaError_t e, const char* what) {
        if (e == cudaSuccess) return true;
        set_error("device key generation: %s: %s", what, cudaGetErrorString(e));
        ok = false;
        return false;
    }
    template <class F>
    bool upload_table(const std::vector<Affine<F>>& t, void*& d, size_t point_bytes) {
        std::vector<uint8_t> packed(t.size() * point_bytes);
        for (size_t i = 0; i < t.size(); i++) pack(packed.data() + i * point_bytes, t[i]);
        // on st and waited for: the kernels run on st, which does not order
        // against a legacy-stream copy
        return check(g16::dev_malloc(&d, packed.size()), "table") &&
               check(cudaMemcpyAsync(d, packed.data(), packed.size(), cudaMemcpyHostToDevice, st), "table upload") &&
               check(cudaStreamSynchronize(st), "table upload");
    }
    bool points(int group, const Fr* k, size_t n, uint8_t* out) {
        const size_t pb = group == 1 ? 64 : 128;
        if (!n) return true;
        if (n * 32 > cap_k) {
            if (d_k) cudaFree(d_k);
            d_k = nullptr;
            cap_k = 0;
            if (!check(g16::dev_malloc(&d_k, n * 32), "scalars")) return false;
            cap_k = n * 32;
        }
        if (n * pb > cap_out) {
            if (d_out) cudaFree(d_out);
            d_out = nullptr;
            cap_out = 0;
            if (!check(g16::dev_malloc(&d_out, n * pb), "points")) return false;
            cap_out = n * pb;
        }
        return check(cudaMemcpyAsync(d_k, k, n * 32, cudaMemcpyHostToDevice, st), "scalar upload") &&
               check(group == 1 ? fixed_base_g1(d_t1, d_k, n, d_out, st) : fixed_base_g2(d_t2, d_k, n, d_out, st),
                     "fixed-base kernels") &&
               check(cudaMemcpyAsync(out, d_out, n * pb, cudaMemcpyDeviceToHost, st), "point readback") &&
               check(cudaStreamSynchronize(st), "synchronize");
    }
};

static std::vector<uint8_t> write_zkey(const g16_synth& s, uint64_t toxic_seed, int threads, int device = -1,
                                       bool* failed = nullptr) {
    host_init();
    SplitMix rng{toxic_seed ^ 0x243F6A8885A308D3ULL};
    const uint32_t n = s.domain, nv = s.n_vars, npub = s.n_public, nc = s.n_constraints;
    int log_n = 0;
    while ((1u << log_n) < n) log_n++;
    Fr omega = domain_root(log_n), shift = domain_root(log_n + 1);
    Fr tau, alpha, beta, delta;
    std::vector<Fr> L(n), den(n), pw(n);
    for (;;) {
        tau = rng.fr_nonzero();
        alpha = rng.fr_nonzero();
        beta = rng.fr_nonzero();
        delta = rng.fr_nonzero();
        // tau must avoid the 2n-th roots of unity
        if (!(tau.pow(std::vector<uint64_t>{2ULL * n, 0, 0, 0}.data(), 4) == Fr::one())) break;
    }
    // L_c(tau) = (tau^n - 1)/n * omega^c / (tau - omega^c)
    uint64_t e_n[4] = {n, 0, 0, 0};
    Fr zt = tau.pow(e_n, 4) - Fr::one();
    Fr factor = zt * Fr::from_u64(n).inv();
    Fr wc = Fr::one();
    for (uint32_t c = 0; c < n; c++) {
        pw[c] = wc;
        den[c] = tau - wc;
        wc = wc * omega;
    }
    auto batch_inv = [](std::vector<Fr>& v) {
        std::vector<Fr> pre(v.size());
        Fr run = Fr::one();
        for (size_t i = 0; i < v.size(); i++) {
            pre[i] = run;
            run = run * v[i];
        }
        Fr iv = run.inv();
        for (size_t i = v.size(); i-- > 0;) {
            Fr x = iv * pre[i];
            iv = iv * v[i];
            v[i] = x;
        }
    };
    batch_inv(den);
    for (uint32_t c = 0; c < n; c++) L[c] = factor * pw[c] * den[c];

    std::vector<Fr> u(nv, Fr::zero()), v(nv, Fr::zero()), wq(nv, Fr::zero());
    for (uint32_t k = 0; k < nc; k++) {
        for (uint32_t t = s.ptr[0][k]; t < s.ptr[0][k + 1]; t++)
            u[s.terms[0][t].sig] = u[s.terms[0][t].sig] + s.terms[0][t].coef * L[k];
        for (uint32_t t = s.ptr[1][k]; t < s.ptr[1][k + 1]; t++)
            v[s.terms[1][t].sig] = v[s.terms[1][t].sig] + s.terms[1][t].coef * L[k];
        wq[1 + s.n_inputs + k] = wq[1 + s.n_inputs + k] + L[k];
    }
    for (uint32_t j = 0; j <= npub; j++) u[j] = u[j] + L[nc + j];

    Fr dinv = delta.inv();
    std::vector<Fr> ic_s(npub + 1), l_s(nv - npub - 1);
    for (uint32_t j = 0; j < nv; j++) {
        Fr x = beta * u[j] + alpha * v[j] + wq[j];
        if (j <= npub) ic_s[j] = x;
        else l_s[j - npub - 1] = x * dinv;
    }
    // H_i = (tau^2n - 1)/(2n) * x_i / (tau - x_i) / delta, x_i = shift * omega^i
    uint64_t e_2n[4] = {2ULL * n, 0, 0, 0};
    Fr factor2 = (tau.pow(e_2n, 4) - Fr::one()) * Fr::from_u64(2ULL * n).inv() * dinv;
    std::vector<Fr> h_s(n);
    Fr xi = shift;
    for (uint32_t i = 0; i < n; i++) {
        pw[i] = xi;
        den[i] = tau - xi;
        xi = xi * omega;
    }
    batch_inv(den);
    for (uint32_t i = 0; i < n; i++) h_s[i] = factor2 * pw[i] * den[i];

    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    FixedBase<Fq> fb1(G1_GENERATOR);
    FixedBase<Fq2> fb2(G2_GENERATOR);
    std::unique_ptr<DevicePoints> dev;
    PointsFn points_of;
    if (device >= 0) {
        dev = std::make_unique<DevicePoints>(device);
        if (!dev->check(cudaSetDevice(device), "cudaSetDevice") ||
            !dev->check(cudaStreamCreateWithFlags(&dev->st, cudaStreamNonBlocking), "stream") ||
            !dev->upload_table(fb1.t, dev->d_t1, 64) || !dev->upload_table(fb2.t, dev->d_t2, 128)) {
            if (failed) *failed = true;
            return {};
        }
        points_of = [&](int group, const Fr* k, size_t n, uint8_t* out) { return dev->points(group, k, n, out); };
    } else {
        points_of = [&](int group, const Fr* k, size_t n, uint8_t* out) {
            if (group == 1) points_into(fb1, k, n, out, 64, threads);
            else points_into(fb2, k, n, out, 128, threads);
            return true;
        };
    }

    BinWriter w;
    w.begin("zkey", 1, 10);
    // 1: protocol
    w.section(1);
    w.u32(1);
    w.end_section();
    // 2: header
    w.section(2);
    w.u32(32);
    w.bytes(FQ_P.p, 32);
    w.u32(32);
    w.bytes(FR_P.p, 32);
    w.u32(nv);
    w.u32(npub);
    w.u32(n);
    uint8_t buf[128];
    auto g1pt = [&](const Fr& k) {
        G1A a = fb1.mul(k).to_affine();
        pack(buf, a);
        w.bytes(buf, 64);
    };
    auto g2pt = [&](const Fr& k) {
        G2A a = fb2.mul(k).to_affine();
        pack(buf, a);
        w.bytes(buf, 128);
    };
    g1pt(alpha);
    g1pt(beta);
    g2pt(beta);
    g2pt(Fr::one());   // gamma = 1
    g1pt(delta);
    g2pt(delta);
    w.end_section();
    // 4: coefficients (double Montgomery)
    w.section(4);
    uint32_t ncoef = (uint32_t)(s.terms[0].size() + s.terms[1].size() + npub + 1);
    w.u32(ncoef);
    auto rec = [&](uint32_t m, uint32_t c, uint32_t sig, const Fr& coef) {
        w.u32(m);
        w.u32(c);
        w.u32(sig);
        Fr stored = Fr::from_std(coef.x.v);   // coef R (Montgomery limbs) -> coef R^2
        w.bytes(stored.x.v, 32);
    };
    for (int m = 0; m < 2; m++)
        for (uint32_t k = 0; k < nc; k++)
            for (uint32_t t = s.ptr[m][k]; t < s.ptr[m][k + 1]; t++) rec(m, k, s.terms[m][t].sig, s.terms[m][t].coef);
    for (uint32_t j = 0; j <= npub; j++) rec(0, nc + j, j, Fr::one());
    w.end_section();
    bool good = true;
    auto point_section = [&](uint32_t id, int group, const std::vector<Fr>& sc) {
        w.section(id);
        size_t at = w.buf.size();
        w.buf.resize(at + sc.size() * (group == 1 ? 64 : 128));
        if (good) good = points_of(group, sc.data(), sc.size(), w.buf.data() + at);
        w.end_section();
    };
    point_section(3, 1, ic_s);
    point_section(9, 1, h_s);
    point_section(8, 1, l_s);
    point_section(5, 1, u);
    point_section(6, 1, v);
    point_section(7, 2, v);
    if (!good) {
        if (failed) *failed = true;
        return {};
    }
    // 10: contributions (empty transcript)
    w.section(10);
    uint8_t zero64[64] = {0};
    w.bytes(zero64, 64);
    w.u32(0);
    w.end_section();
    return std::move(w.buf);
}

static std::vector<uint8_t> write_r1cs(const g16_synth& s) {
    host_init();
    BinWriter w;
    w.begin("r1cs", 1, 3);
    w.section(1);
    w.u32(32);
    w.bytes(FR_P.p, 32);
    w.u32(s.n_vars);
    w.u32(0);                          // nOutputs
    w.u32(s.n_public);                 // nPubInputs
    w.u32(s.n_inputs - s.n_public);    // nPrvInputs
    w.u64(s.n_vars);                   // nLabels
    w.u32(s.n_constraints);
    w.end_section();
    w.section(2);
    auto lc = [&](const Term* t, uint32_t cnt) {
        w.u32(cnt);
        for (uint32_t i = 0; i < cnt; i++) {
            w.u32(t[i].sig);
            uint64_t v[4];
            t[i].coef.to_std(v);
            w.bytes(v, 32);
        }
    };
    Term c_term;
    c_term.coef = Fr::one();
    for (uint32_t k = 0; k < s.n_constraints; k++) {
        lc(&s.terms[0][s.ptr[0][k]], s.ptr[0][k + 1] - s.ptr[0][k]);
        lc(&s.terms[1][s.ptr[1][k]], s.ptr[1][k + 1] - s.ptr[1][k]);
        c_term.sig = 1 + s.n_inputs + k;
        lc(&c_term, 1);
    }
    w.end_section();
    w.section(3);
    for (uint64_t i = 0; i < s.n_vars; i++) w.u64(i);
    w.end_section();
    return std::move(w.buf);
}

extern "C" {

int g16_synth_new(uint64_t seed, uint32_t n_constraints, uint32_t n_inputs, uint32_t n_public, g16_synth** out) {
    if (!out || n_constraints == 0 || n_public > n_inputs || n_inputs == 0) {
        set_error("g16_synth_new: need n_constraints > 0 and 0 < n_public <= n_inputs");
        return G16_ERR_INVALID_ARGUMENT;
    }
    host_init();
    uint64_t total = (uint64_t)n_constraints + n_public;
    int p = 0;
    while ((1ULL << (p + 1)) <= total) p++;
    if (p + 1 > 27) {
        set_error("g16_synth_new: domain 2^%d exceeds 2^27", p + 1);
        return G16_ERR_INVALID_ARGUMENT;
    }
    auto s = std::make_unique<g16_synth>();
    s->n_constraints = n_constraints;
    s->n_inputs = n_inputs;
    s->n_public = n_public;
    s->n_vars = 1 + n_inputs + n_constraints;
    s->domain = 1u << (p + 1);
    build_structure(*s, seed);
    *out = s.release();
    return G16_OK;
}

int g16_synth_zkey_device(const g16_synth* cs, uint64_t toxic_seed, int device, uint8_t* out, size_t cap,
                          size_t* len_out) {
    if (!cs || !len_out || device < 0) {
        set_error("g16_synth_zkey_device: null argument or negative device");
        return G16_ERR_INVALID_ARGUMENT;
    }
    g16_synth* s = const_cast<g16_synth*>(cs);
    std::lock_guard<std::mutex> g(s->mu);
    if (!s->cached || s->cached_seed != toxic_seed) {
        bool failed = false;
        std::vector<uint8_t> z = write_zkey(*s, toxic_seed, 0, device, &failed);
        if (failed) return G16_ERR_DEVICE;
        s->zkey = std::move(z);
        s->cached = true;
        s->cached_seed = toxic_seed;
    }
    *len_out = s->zkey.size();
    if (!out) return G16_OK;
    if (cap < s->zkey.size()) {
        set_error("g16_synth_zkey_device: buffer of %zu bytes, need %zu", cap, s->zkey.size());
        return G16_ERR_INVALID_ARGUMENT;
    }
    std::memcpy(out, s->zkey.data(), s->zkey.size());
    std::vector<uint8_t>().swap(s->zkey);
    s->cached = false;
    return G16_OK;
}

void g16_synth_free(g16_synth* s) { delete s; }
uint32_t g16_synth_n_vars(const g16_synth* s) { return s ? s->n_vars : 0; }
uint32_t g16_synth_domain_size(const g16_synth* s) { return s ? s->domain : 0; }

int g16_synth_witness(const g16_synth* s, uint64_t witness_seed, uint8_t* out_mont) {
    if (!s || !out_mont) return G16_ERR_INVALID_ARGUMENT;
    std::vector<Fr> w;
    compute_witness(*s, witness_seed, w);
    for (size_t i = 0; i < w.size(); i++) std::memcpy(out_mont + 32 * i, w[i].x.v, 32);
    return G16_OK;
}

int g16_synth_zkey(const g16_synth* cs, uint64_t toxic_seed, int threads, uint8_t* out, size_t cap,
                   size_t* len_out) {
    if (!cs || !len_out) return G16_ERR_INVALID_ARGUMENT;
    g16_synth* s = const_cast<g16_synth*>(cs);
    std::lock_guard<std::mutex> g(s->mu);
    if (!s->cached || s->cached_seed != toxic_seed) {
        s->zkey = write_zkey(*s, toxic_seed, threads);
        s->cached = true;
        s->cached_seed = toxic_seed;
    }
    *len_out = s->zkey.size();
    if (!out) return G16_OK;
    if (cap < s->zkey.size()) {
        set_error("g16_synth_zkey: buffer of %zu bytes, need %zu", cap, s->zkey.size());
        return G16_ERR_INVALID_ARGUMENT;
    }
    std::memcpy(out, s->zkey.data(), s->zkey.size());
    // the copy is the caller's now; release the cached one
    std::vector<uint8_t>().swap(s->zkey);
    s->cached = false;
    return G16_OK;
}

int g16_synth_r1cs(const g16_synth* s, uint8_t* out, size_t cap, size_t* len_out) {
    if (!s || !len_out) return G16_ERR_INVALID_ARGUMENT;
    std::vector<uint8_t> b = write_r1cs(*s);
    *len_out = b.size();
    if (!out) return G16_OK;
    if (cap < b.size()) return G16_ERR_INVALID_ARGUMENT;
    std::memcpy(out, b.data(), b.size());
    return G16_OK;
}

}  // extern "C"

// ---- seeded inputs for the standalone MSM workloads ----
extern "C" {

// n affine points k_i G (G1: group 1, 64 B each; G2: group 2, 128 B each),
// k_i uniform in [1, r) from the seed.
int g16_synth_points(int group, uint64_t seed, size_t n, int threads, uint8_t* out) {
    if (!out || (group != 1 && group != 2)) {
        set_error("g16_synth_points: group must be 1 or 2 and out non-null");
        return G16_ERR_INVALID_ARGUMENT;
    }
    host_init();
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    SplitMix rng{seed ^ 0x452821E638D01377ULL};
    std::vector<Fr> k(n);
    for (size_t i = 0; i < n; i++) k[i] = rng.fr_nonzero();
    if (group == 1) {
        FixedBase<Fq> fb(G1_GENERATOR);
        points_into(fb, k.data(), n, out, 64, threads);
    } else {
        FixedBase<Fq2> fb(G2_GENERATOR);
        points_into(fb, k.data(), n, out, 128, threads);
    }
    return G16_OK;
}

// n scalars in standard form: dist 0 = uniform in [0, r); dist 1 = 35% zero,
// 35% one, 30% uniform.
int g16_synth_scalars(uint64_t seed, size_t n, int dist, uint8_t* out_std) {
    if (!out_std || (dist != 0 && dist != 1)) {
        set_error("g16_synth_scalars: dist must be 0 or 1 and out non-null");
        return G16_ERR_INVALID_ARGUMENT;
    }
    host_init();
    SplitMix rng{seed ^ 0xBE5466CF34E90C6CULL};
    for (size_t i = 0; i < n; i++) {
        uint64_t v[4] = {0, 0, 0, 0};
        double u = dist ? rng.uniform() : 1.0;
        if (u < 0.35) {
        } else if (u < 0.70) {
            v[0] = 1;
        } else {
            uint64_t x[4] = {rng.next(), rng.next(), rng.next(), rng.next() & ((1ULL << 62) - 1)};
            if (geq4(x, FR_P.p)) sub4(x, x, FR_P.p);
            std::memcpy(v, x, 32);
        }
        std::memcpy(out_std + 32 * i, v, 32);
    }
    return G16_OK;
}

}  // extern "C"
