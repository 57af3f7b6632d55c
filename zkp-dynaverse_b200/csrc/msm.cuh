// Pippenger multi-scalar multiplication on sm_100a for BN254 G1 and G2.
//
// One engine serves the plain MSM (OperatorBackend::msm / msm_g2_host,
// crates/protocol/src/types.rs:295-356), the padded batch
// (dvgpu_bn254_msm_batch, native/src/icicle_msm.cu:810-880), uneven batches
// and the sparse-index MSM (types.rs:262-345): every input is a list of
// "sets" (independent MSMs) over concatenated point/scalar arrays, and the
// set index is folded into the bucket key, so all sets run in the same
// launches.
//
// Pipeline (all on one stream):
//   1. hist     signed c-bit digits of every scalar, count per (set, window, bucket)
//   2. scan     exclusive prefix sum -> bucket offsets in the sorted list
//   3. scatter  counting-sort placement of (point index | sign) per digit
//   4. accum    persistent, perfectly balanced bucket accumulation: each thread
//               sums a fixed-length slice of the sorted list with XYZZ mixed
//               additions; buckets cut by a slice boundary leave partials
//   5. fixup    partial sums of buckets that span slices are merged
//   6. segments per (set, window): running sums over segments of 2^seg_log buckets
//   7. wlevel   logarithmic-depth levels of the weighted bucket sum (suffix
//               scan + tree per block), down to one value per (set, window)
//   8. host     Horner over the windows and normalisation to affine
// With a table of precomputed window multiples (resident bases), steps 1-7
// use one bucket set per MSM and step 8 only normalises.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "curve.cuh"
#include "engine.hpp"

namespace dv {

struct MsmPlan {
    int c;            // window width in bits
    int windows;      // ceil(255 / c): top window never carries out
    uint32_t buckets; // 2^(c-1) signed-digit buckets per window
    int seg_log;      // bucket-reduction segment length = 2^seg_log
    int seg_force = 0;  // > 0: this segment length (log2) instead of msm_seg_log's
};

// Bucket-reduction segment length (log2) for a launch of all_buckets
// buckets, `buckets` per window set, window width c.
int msm_seg_log(uint64_t all_buckets, uint32_t buckets, int c, bool g1);

// Cost model: windows * (10 * n + 28 * buckets) base-field multiplications
// (XYZZ mixed add = 10, two full adds per bucket in the reduction = 28).
MsmPlan msm_plan(uint64_t points_per_set, int force_c);

// Optional per-phase device timing (CUDA events on the launching stream).
// Phases: 0 hist, 1 scan, 2 scatter, 3 accumulation, 4 split-bucket merges,
// 5 bucket reduction, 6 unused, 7 window D2H + host Horner.
enum { MSM_PHASES = 8 };
struct MsmTimeline {
    bool enabled = false;
    cudaEvent_t ev[7] = {};
    cudaEvent_t acc_ev[4] = {};
    double ms[MSM_PHASES] = {};
    uint64_t calls = 0;
    uint64_t accum_mixed_adds = 0;  // N * windows summed over timed calls (for the roofline)
};

struct MsmWorkspace {
    DevBuf set_off, counts, offsets, cursor, scan_tiles, sorted, buckets, pgid, ppt, fix_list, fix_count, segs, windows,
        err;
    DevBuf sd_jobs, sd_req, sd_partial, sd_out;  // direct small sparse MSMs
    PinnedBuf host_windows, host_err, host_desc;
    MsmTimeline timeline;
};

struct MsmStats {
    uint64_t calls = 0, sets = 0, points = 0, last_c = 0;
};

// Precomputed window multiples of a fixed base set (a resident SRS):
// table[i * windows + w] = 2^(c w) P_i.  With a table, every window of an MSM
// adds into one shared bucket set and no window combination is needed.
template <class F>
struct MsmPrecomp {
    const Affine<F>* table;
    int c;
    int windows;
};

// d_points: Montgomery-form affine points, d_scalars: canonical 8-word
// little-endian scalars (checked < r), both concatenated over sets.
// set_offsets (host, count + 1 entries) delimit the sets.  host_out receives
// count canonical affine points (2 * sizeof(F) bytes each, all-zero for
// infinity).  Throws InvalidArgument for non-canonical scalars.
// Sparse MSMs over a resident table of window multiples, summed directly:
// each (entry, window) term d T is formed by one thread (double-and-add on
// the signed c-bit digit d), then block and request sums.  For small
// supports, where the bucket pipeline's launch chain dominates.  d_idx:
// entry base indices (checked < nbases), d_vals: canonical scalars (checked),
// offs (host, count + 1): entries of each request.  host_out: count
// canonical affine G1 points.  Throws InvalidArgument as msm_run does.
void msm_sparse_direct(MsmWorkspace& ws, const MsmPrecomp<Fq>& pre, uint64_t nbases, const uint64_t* d_idx,
                       const uint32_t* d_vals, const uint32_t* offs, uint32_t count, uint8_t* host_out,
                       cudaStream_t stream);
// Terms (entries x windows) up to which sparse calls take the direct path:
// with a c = 8 table (32 windows) the direct path wins up to 2048 entries
// (k = 1024: 0.29 against 0.73 ms; 2048: 0.48 against 0.71 ms) and the
// bucket pipeline from 3072 (0.46 against 0.67 ms).
constexpr uint64_t SPARSE_DIRECT_MAX_TERMS = 1u << 16;

template <class F>
void msm_run(MsmWorkspace& ws, const Affine<F>* d_points, const uint32_t* d_scalars, const uint32_t* set_offsets,
             uint32_t count, int force_c, cudaStream_t stream, uint8_t* host_out, MsmStats* stats,
             const MsmPrecomp<F>* pre = nullptr);

// How the digits of one launch sequence map to sets, scalars and points.
// Digit i (0 <= i < off[count]) belongs to the set k with
// off[k] <= i < off[k + 1]; its scalar is src[k] + (i - off[k]) (i itself
// when src is null); its point is i - off[k] with prefix (every set uses a
// prefix of one base array), else the scalar's index.  With per-term arrays
// (term_point, term_scalar, device, off[count] entries each) term i takes
// point term_point[i] and scalar term_scalar[i] instead: the sets of one
// launch can then draw entries from anywhere in a base array (or its table)
// and share scalars, with no gathered copy.
struct SetMap {
    const uint32_t* off;  // device, count + 1 entries
    const uint32_t* src;  // device or null
    uint32_t count;
    int prefix;
    const uint32_t* term_point = nullptr;
    const uint32_t* term_scalar = nullptr;
};

// Window plan of a launch sequence of count sets (largest max_set, total
// points in all): force_c, else a cost model that charges every set its
// windows * 2^(c-1) buckets, bounded so that count * windows * buckets stays
// launchable; a precomputed table fixes c and uses one bucket set per MSM.
template <class F>
MsmPlan msm_plan_batch(uint32_t count, uint32_t max_set, uint64_t total, int force_c, const MsmPrecomp<F>* pre);

// The device part of an MSM launch sequence: digit sort, accumulation,
// merges and bucket reduction, all on `stream`, without host
// synchronisation.  Leaves count * (pre ? 1 : windows) XYZZ window sums in
// ws.windows and the lowest non-canonical scalar index (or 0xffffffff) in
// *d_err, which the caller initialises.  Allocates only when a workspace
// buffer must grow, so a second call with the same shapes allocates nothing
// (and can be captured in a CUDA graph).
template <class F>
void msm_enqueue(MsmWorkspace& ws, const Affine<F>* d_points, const uint32_t* d_scalars, const SetMap& map,
                 uint32_t n, const MsmPlan& plan, const MsmPrecomp<F>* pre, uint32_t* d_err, cudaStream_t stream);

// Device tail: Horner over each set's window sums (weights 2^(c w)) and
// normalisation to canonical affine bytes (2 * sizeof(F) per set, all-zero
// for infinity), one thread per set.  Set k is written at result position
// d_out_idx[k] (k when null).
template <class F>
void msm_finish_device(const XYZZ<F>* d_windows, uint32_t count, int windows_per_set, int c, const uint32_t* d_out_idx,
                       uint8_t* d_out, cudaStream_t stream);

// Builds the table of precomputed window multiples (windows * n entries).
template <class F>
void msm_precompute(const Affine<F>* d_bases, uint64_t n, int c, int windows, Affine<F>* d_table, cudaStream_t stream);
// Window width for a precomputed table of n bases (cost model).
MsmPlan msm_plan_precomputed(uint64_t n);

// Canonical bytes -> Montgomery affine, with canonical and on-curve checks.
// Sets *first_bad (device) to the lowest failing index, or leaves it.
template <class F>
void convert_points(const uint8_t* d_canon, Affine<F>* d_out, uint64_t n, uint32_t* d_first_bad, cudaStream_t stream);

// Gather of a table of window multiples (W entries per base):
// out[j W + w] = table[idx[j] W + w], idx checked against nbases.
template <class F>
void gather_table(const Affine<F>* d_table, uint64_t nbases, int W, const uint64_t* d_idx, uint64_t k,
                  Affine<F>* d_out, uint32_t* d_first_bad, cudaStream_t stream);

// Gather (sparse MSM): out[j] = bases[idx[j]], with idx checked against nbases.
template <class F>
void gather_points(const Affine<F>* d_bases, uint64_t nbases, const uint64_t* d_idx, uint64_t k, Affine<F>* d_out,
                   uint32_t* d_first_bad, cudaStream_t stream);

}  // namespace dv
