// BN254 Fr number-theoretic transform on sm_100a.
//
// Semantics follow ark-poly 0.4 Radix2EvaluationDomain as used by the
// reference CPU path (crates/gpu/src/lib.rs:99-118,
// crates/protocol/src/dynaverse.rs:1157-1164) and the ICICLE wrapper
// (crates/gpu/src/icicle.rs:429-456): natural order in and out, forward =
// evaluations at w^i, inverse = coefficients scaled by 1/n, w = the 2^28-th
// root GENERATOR^((r-1)/2^28) (GENERATOR = 5) squared down to order n.
// Coset forms use the offset g = 5: forward scales coefficient j by g^j
// before the transform, inverse scales output i by g^-i after it.
//
// Layout: canonical little-endian 32-byte elements in HBM (the wire format).
// Values stay canonical throughout: every multiplier (twiddles, coset and
// scale factors) is held in Montgomery form, and mont_mul(a, x R) = a x.
// The transform is decimation-in-frequency radix-2, grouped into passes of
// up to 11 stages; each pass stages a tile of 2^11 elements (one group of
// 2^k elements with stride 2^lb, or several consecutive groups when k < 11)
// in shared memory as two swizzled planes of 16-byte halves and runs its
// stages in register rounds of two (each thread owns 4 elements per round),
// with twiddles from a resident table w^i (i < n/2).  The last pass writes
// the output in natural order (bit reversal fused with the inverse and
// coset scaling).
//
// Batches of transforms of any sizes run as ONE persistent launch: blocks
// take tiles from an atomic counter in pass order; a tile of pass p of a
// transform waits (bounded) until every tile of its pass p - 1 is done.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <vector>

#include "curve.cuh"
#include "engine.hpp"

namespace dv {

enum NttKind { NTT_FORWARD = 0, NTT_INVERSE = 1, NTT_COSET_FORWARD = 2, NTT_COSET_INVERSE = 3 };

struct NttTables {
    DevBuf tw;         // w^i, i < n/2 (Montgomery), w of order n (or w^-1 for inverse)
    DevBuf pre_hi, pre_lo, post_hi, post_lo;  // two-level scaling tables
    DevBuf consts;     // per-(size, kind) field constants
    int split = 0;     // bits in the low table index
    DevBuf glv;        // G1 transform: GLV halves of every twiddle and of 1/n (ecntt.cu)
    int glv_ready = 0;
};

struct NttWorkspace {
    DevBuf work;
    DevBuf err;
    std::map<int, std::unique_ptr<NttTables>> tables;  // key: logn * 4 + kind
    uint64_t calls = 0, elements = 0;
};

constexpr int NTT_MAX_LOG = 26;

// d_in, d_out: canonical elements (may alias).  Throws InvalidArgument for
// non-canonical input (checked on device, reported after the transform).
void ntt_run(NttWorkspace& ws, const uint8_t* d_in, uint8_t* d_out, int logn, int kind, cudaStream_t stream);

// Twiddle and scaling tables of one (size, kind), built on first use and
// kept in the workspace.
NttTables& ntt_tables(NttWorkspace& ws, int logn, int kind, cudaStream_t stream);
// 1/n of a table set as a canonical scalar (8 little-endian words), on the device.
const uint32_t* ntt_ninv_canonical(NttTables& tables);

// G1 transform of rows x 2^logn XYZZ points held in `work` (overwritten):
// natural-order results (x 1/n for the inverse) in `out` (ecntt.cu).
void g1_ntt_rows_xyzz(NttWorkspace& ws, XYZZ<Fq>* work, int logn, uint64_t rows, bool inverse, XYZZ<Fq>* out,
                      cudaStream_t stream);

// ---------------------------------------------------------------- batches
struct NttBatchItem {
    const uint8_t* in;  // canonical elements on the device
    uint8_t* out;       // may alias in
    int logn;           // 1..24
    int kind;           // NttKind
};

// A prepared batch: descriptors, the tile list and per-transform working
// vectors on the device.  Prepare once, enqueue any number of times (each
// enqueue = two memsets and one kernel launch, no allocation, no host
// synchronisation: capturable in a CUDA graph).
// Elements per tile of the batched NTT: 2^tile_log, staged in 32 << tile_log
// bytes of shared memory (2^11: 64 KB, three blocks per SM).
constexpr int BATCH_TILE_MIN = 8, BATCH_TILE_DEFAULT = 11, BATCH_TILE_MAX = 12;
struct NttBatch {
    DevBuf descs, tiles, ctl, work, errs;
    uint32_t count = 0, ntiles = 0, grid = 0;
    int radix_log = 2;  // register round of the kernel: radix 2, 4 or 8
    int tile_log = BATCH_TILE_DEFAULT;
    uint64_t elements = 0;
    std::vector<uint64_t> work_off;
};
void ntt_batch_prepare(NttWorkspace& ws, NttBatch& batch, const std::vector<NttBatchItem>& items,
                       cudaStream_t stream, int tile_log = BATCH_TILE_DEFAULT);
void ntt_batch_enqueue(NttBatch& batch, cudaStream_t stream);
// Selects the kernel's register round (radix_log 1, 2 or 3: radix 2, 4 or
// 8 butterflies per round) and sizes the persistent grid from that
// kernel's occupancy.  Every radix computes the same bytes.
void ntt_batch_set_radix(NttBatch& batch, int radix_log);
// After the stream has completed: throws InvalidArgument naming the first
// transform with a non-canonical input, or CudaFailure if a dependency wait
// gave up.
void ntt_batch_check(NttBatch& batch, cudaStream_t stream);

}  // namespace dv
