// Stage 0 of the prover, one constraint row: A[row] = sum over the CSR row of
// coefficient * witness, the same for B, and C = A * B (CpuCircuit::gather,
// crates/groth16/src/cpu.rs:140-174, and compute_h, :316-341).  Zero witness
// values are skipped and ones added without a product, which is exact either
// way (cpu.rs:150-170).
#pragma once
#include "field.cuh"

namespace g16d {

__device__ __forceinline__ void gather_row(uint32_t row, const uint32_t* __restrict__ rpa,
                                           const uint32_t* __restrict__ siga, const uint32_t* __restrict__ vida,
                                           const uint32_t* __restrict__ rpb, const uint32_t* __restrict__ sigb,
                                           const uint32_t* __restrict__ vidb, const uint4* __restrict__ values,
                                           const uint4* __restrict__ w, uint4* __restrict__ A, uint4* __restrict__ B,
                                           uint4* __restrict__ C) {
    Fr acc[2];
    const uint32_t* rp[2] = {rpa, rpb};
    const uint32_t* sg[2] = {siga, sigb};
    const uint32_t* vd[2] = {vida, vidb};
#pragma unroll
    for (int m = 0; m < 2; m++) {
        Fr a = Fr::zero();
        for (uint32_t k = rp[m][row]; k < rp[m][row + 1]; k++) {
            Fr wv = load32(reinterpret_cast<const Fr*>(w) + sg[m][k]);
            if (wv.is_zero()) continue;
            Fr v = load32(reinterpret_cast<const Fr*>(values) + vd[m][k]);
            a = add(a, wv.is_one() ? v : mul(v, wv));
        }
        acc[m] = a;
    }
    store32(reinterpret_cast<Fr*>(A) + row, acc[0]);
    store32(reinterpret_cast<Fr*>(B) + row, acc[1]);
    store32(reinterpret_cast<Fr*>(C) + row, mul(acc[0], acc[1]));
}

}  // namespace g16d
