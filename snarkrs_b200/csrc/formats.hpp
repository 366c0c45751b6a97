// snarkjs binfile formats (.zkey, .wtns, .r1cs): host-side structures.
#pragma once
#include <cstdint>
#include <cstring>
#include <vector>
#include "host_bn254.hpp"

#include "g16b200.h"

namespace g16 {

// A parsed proving key (ProvingKey, crates/formats/src/lib.rs:35-65).
struct ZkeyHost {
    uint32_t n_vars = 0, n_public = 0, domain_size = 0;
    std::vector<uint8_t> alpha_g1, beta_g1, beta_g2, gamma_g2, delta_g1, delta_g2, ic;
    std::vector<uint32_t> row_ptr[2], signal[2], value_id[2];
    std::vector<uint8_t> values;   // interned Fr, Montgomery, 32 bytes each
    std::vector<uint8_t> a_query, b_g1_query, b_g2_query, l_query, h_query;
    uint32_t h_basis = 0;   // 0 snarkjs odd coset (domain_size H bases), 1 gnark bit-reversed (domain_size - 1)
};

int zkey_parse(const uint8_t* d, size_t len, bool check_points, ZkeyHost& k);
// gnark v0.14 proving-key dump + verifying key (gnark.cpp): a key with the gnark
// H basis and no constraint matrices
int gnark_key_parse(const uint8_t* pk, size_t pk_len, const uint8_t* vk, size_t vk_len, ZkeyHost& k);
// gnark witness dump: W, A.w, B.w (Montgomery Fr bytes)
int gnark_witness_parse(const uint8_t* d, size_t len, std::vector<uint8_t> out[3]);
void zkey_view(const ZkeyHost& k, g16_zkey_view& v);
int wtns_parse(const uint8_t* d, size_t len, std::vector<uint8_t>& out_mont);
std::vector<uint8_t> wtns_write(const uint8_t* w_mont, size_t n);

// iden3 binfile writer
struct BinWriter {
    std::vector<uint8_t> buf;
    size_t sec_start = 0;
    void begin(const char* magic, uint32_t version, uint32_t nsec);
    void section(uint32_t id);
    void end_section();
    void u32(uint32_t x) { bytes(&x, 4); }
    void u64(uint64_t x) { bytes(&x, 8); }
    void bytes(const void* p, size_t n) {
        const uint8_t* b = (const uint8_t*)p;
        buf.insert(buf.end(), b, b + n);
    }
};

}  // namespace g16
