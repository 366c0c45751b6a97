// Host BN254 constants and helpers (see host_bn254.hpp).
#include "host_bn254.hpp"
#include <mutex>
#include <vector>

namespace g16 {

G1A G1_GENERATOR;
G2A G2_GENERATOR;
Fq2 TWIST_B;

static Fq fq_dec(const char* s) {
    uint64_t v[4] = {0, 0, 0, 0};
    for (; *s; s++) {
        u128 carry = (unsigned)(*s - '0');
        for (int i = 0; i < 4; i++) {
            u128 t = (u128)v[i] * 10 + carry;
            v[i] = (uint64_t)t;
            carry = t >> 64;
        }
    }
    return Fq::from_std(v);
}

void host_init() {
    static std::once_flag once;
    std::call_once(once, [] {
        G1_GENERATOR.x = Fq::from_u64(1);
        G1_GENERATOR.y = Fq::from_u64(2);
        G1_GENERATOR.inf = false;
        // the standard BN254 G2 generator (EIP-197)
        G2_GENERATOR.x = {fq_dec("10857046999023057135944570762232829481370756359578518086990519993285655852781"),
                          fq_dec("11559732032986387107991004021392285783925812861821192530917403151452391805634")};
        G2_GENERATOR.y = {fq_dec("8495653923123431417604973247489272438418190587263600148770280649306958101930"),
                          fq_dec("4082367875863433681332203403145435568316851327593401208105741076214120093531")};
        G2_GENERATOR.inf = false;
        Fq2 xi = {Fq::from_u64(9), Fq::one()};
        TWIST_B = Fq2{Fq::from_u64(3), Fq::zero()} * xi.inv();
    });
}

Fr domain_root(int log_n) {
    uint64_t e[4];
    std::memcpy(e, FR_P.p, 32);
    e[0] -= 1;
    for (int k = 0; k < 28; k++)
        for (int i = 0; i < 4; i++) e[i] = (e[i] >> 1) | (i < 3 ? (e[i + 1] << 63) : 0);
    Fr w = Fr::from_u64(5).pow(e, 4);
    for (int i = log_n; i < 28; i++) w = w.sqr();
    return w;
}

template <class F>
void batch_to_affine(const Jac<F>* in, Affine<F>* out, size_t n) {
    std::vector<F> acc(n);
    F run = F::one();
    for (size_t i = 0; i < n; i++) {
        acc[i] = run;
        if (!in[i].is_inf()) run = run * in[i].z;
    }
    F inv = run.inv();
    for (size_t i = n; i-- > 0;) {
        if (in[i].is_inf()) {
            out[i].x = F::zero();
            out[i].y = F::zero();
            out[i].inf = true;
            continue;
        }
        F zi = inv * acc[i];
        inv = inv * in[i].z;
        F zi2 = zi.sqr();
        out[i].x = in[i].x * zi2;
        out[i].y = in[i].y * zi2 * zi;
        out[i].inf = false;
    }
}

template void batch_to_affine<Fq>(const Jac<Fq>*, Affine<Fq>*, size_t);
template void batch_to_affine<Fq2>(const Jac<Fq2>*, Affine<Fq2>*, size_t);

}  // namespace g16
