// Host optimal-ate pairing over BN254 and the Groth16 verifier built on it.
//
// Replaces the reference's verify::verify / verify_unchecked / check_proof /
// aggregate_public (crates/groth16/src/verify.rs:49-175), which prove::prove
// runs on every proof before returning it (crates/groth16/src/prove.rs:34-92).
// A verification is four Miller loops, one host thread each, whose product
// goes through one final exponentiation, with B's subgroup check on a fifth
// thread: a few milliseconds of host time.  It never runs on the device.
//
// Tower: Fq2 = Fq[u]/(u^2 + 1), Fq6 = Fq2[v]/(v^3 - xi) with xi = 9 + u,
// Fq12 = Fq6[w]/(w^2 - v).  G2 lives on the D-type sextic twist
// y^2 = x^3 + 3/xi, mapped into E(Fq12) by (x, y) -> (x w^2, y w^3).
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include "host_bn254.hpp"

namespace g16 {

struct VerifyingKey {
    G1A alpha1;
    G2A beta2, gamma2, delta2;
    const G1A* ic = nullptr;   // n_ic points: the constant wire, then one per public input
    size_t n_ic = 0;
};

enum class VerifyResult { Ok, PublicInputCount, EmptyKey, UnsafeKey, InvalidProof, PairingFailed };

// verify::verify: key structure, proof elements (on curve, B in the r-order
// subgroup, none at infinity), then the pairing equation
//   e(-A, B) e(alpha, beta) e(L, gamma) e(C, delta) = 1,  L = IC0 + sum w_i IC_i.
// public_mont: n_public Montgomery Fr.  why receives a one-line reason.
VerifyResult groth16_verify(const VerifyingKey& vk, const uint8_t* public_mont, size_t n_public, const G1A& a,
                            const G2A& b, const G1A& c, std::string* why);

// prod_i e(P_i, Q_i) == 1 for affine points (pairs with a point at infinity
// contribute 1).  For the tests of the pairing itself.
bool pairing_product_is_one(const G1A* p, const G2A* q, size_t n);

}  // namespace g16
