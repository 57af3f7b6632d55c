// Batched G2 wire validation and fixed-base SRS generation on sm_100a.
//
// G2 validation follows the reference's parser and predicates
// (native/include/icicle_g2_wire.cuh:17-32, native/src/icicle_g2_validation.cu:20-71,
// crates/gpu/src/g2_validation.rs:243-299): per point a mask with bit 1 =
// bad encoding / non-canonical field, 2 = off curve, 4 = outside the
// order-r subgroup; algorithm 1 = [r]P == 0, 2 = psi(P) == [6x^2]P,
// 3 = [x]P + P + psi([x]P) + psi^2([x]P) == 2 psi^3([x]P)  (x = BN seed).
// One launch covers any number of points (the reference chunks at 4096).
//
// Fixed base follows native/include/icicle_setup.cuh:44-112: a resident
// table [d * 16^w] G (64 windows x 16 digits, affine, Montgomery) and one
// thread per scalar summing 64 table entries; normalisation to affine uses
// one field inversion per warp (Montgomery's trick over warp shuffles).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/dynaverse_gpu.h"
#include "curve.cuh"
#include "engine.hpp"

namespace dv {

struct G2CheckAccum {
    unsigned long long invalid;
    unsigned long long first;
    uint32_t mask;
    uint32_t pad;
};

// wire: device bytes (n * 128); masks: device u32[n]; acc: device accumulator.
void g2_check_launch(const uint8_t* d_wire, uint64_t n, uint32_t algorithm, uint32_t* d_masks, G2CheckAccum* d_acc,
                     cudaStream_t stream, unsigned threads = 128);
// Attributes and theoretical occupancy of the check kernel at a block size,
// and of the checked fixed-base generation (whose normalisation is fused).
void g2_kernel_resources(unsigned threads, DvgpuG2KernelResources& out);

struct FixedBaseTables {
    DevBuf g1, g2;  // 16 * 2^15 affine entries each: |d| 2^(16 w) G
    DevBuf bases;   // the 16 window bases while a table is built
    bool g1_ready = false, g2_ready = false;
};

// scalars: device canonical; out: device canonical affine bytes (64 / 128 each).
void fixed_base_launch(FixedBaseTables& tabs, const uint8_t* d_scalars, uint64_t n, int g2, uint8_t* d_out,
                       uint32_t* d_first_bad, cudaStream_t stream);
// The smallest index of a non-canonical scalar into d_first_bad (atomicMin).
void fixed_base_validate(const uint8_t* d_scalars, uint64_t n, uint32_t* d_first_bad, cudaStream_t stream);
// Entries of one fixed-base table (16 windows of 2^15 multiples).
uint64_t fixed_base_table_entries();

}  // namespace dv
