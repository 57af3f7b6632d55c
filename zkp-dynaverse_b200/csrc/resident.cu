// Resident transactional buffers (the RebuildBackend of the reference).
//
// Semantics follow the CPU reference CpuRebuildBackend
// (crates/protocol/src/incremental_rebuild/operators.rs:52-111, 113-500) and
// the op encoding of its native binding (crates/gpu/src/resident.rs:250-402,
// native/include/dynaverse_gpu.h:100-160):
//   - buffers of Fr or G1 elements, allocated (zero / infinity) before seal;
//     after seal only writable buffers accept writes; registered MSM bases
//     are immutable and only READ and MSM_G1 accept them;
//   - one transaction at a time: the first write to an element saves its
//     old value in the undo journal, rollback restores every saved element,
//     commit publishes;
//   - operations: write/read, copy, reverse copy, transpose (optionally
//     scaled by root^(row col)), row transforms (Fr NTT or G1 transform),
//     complete transforms of one packet, field zip (add/sub/mul), point
//     scaling, MSMs over resident buffers (G1) or host bases (G2).
//
// Device layout: Fr elements as canonical 8 x u32 words (32 B), G1 elements
// as XYZZ points in Montgomery form (128 B; all-zero = infinity), registered
// bases as Montgomery affine points (64 B).  The journal is a fixed device
// arena of records (buffer, element, old bytes); each element carries the
// epoch of the transaction that last saved it, so "saved in this
// transaction" is one compare and commit needs no device work.
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "abi_util.hpp"
#include "backend.hpp"

namespace dv {

bool root_order_2_20(const uint8_t* root);

namespace {

enum Opcode : uint32_t {
    OP_ALLOC = 1, OP_LENGTH, OP_KIND, OP_BEGIN, OP_ROLLBACK, OP_WRITE, OP_READ, OP_COPY, OP_REVERSE, OP_TRANSPOSE,
    OP_TRANSFORM, OP_ZIP, OP_SCALE, OP_MSM_G1, OP_MSM_G2, OP_ALLOC_BASES, OP_TRANSFORM_PACKET
};
enum Kind : uint32_t { KIND_FR = 0, KIND_G1 = 1, KIND_BASES = 2 };

constexpr uint32_t RECORD_BYTES = 144;  // 16-byte header + up to 128 bytes of element
constexpr uint64_t MAX_PACKET = 4096;

uint32_t elem_bytes(uint32_t kind) { return kind == KIND_FR ? 32u : kind == KIND_G1 ? 128u : 64u; }

// ----------------------------------------------------------------- kernels
// Journal the elements dst[index(i)] for i < n (index = offset + i, or the
// transpose target col * rows + row of i = start + i) whose epoch marker is
// not the current transaction's.
__global__ void k_journal(uint8_t* __restrict__ data, uint32_t* __restrict__ marks, uint32_t esize, uint32_t buf,
                          uint64_t offset, uint64_t n, uint64_t rows, uint64_t cols, int transpose, uint32_t epoch,
                          uint8_t* __restrict__ arena, uint32_t capacity, uint32_t* __restrict__ ctl) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t e = offset + i;
    if (transpose) e = (e % cols) * rows + e / cols;
    if (marks[e] == epoch) return;
    marks[e] = epoch;
    const uint32_t slot = atomicAdd(ctl, 1u);
    if (slot >= capacity) {
        atomicOr(ctl + 1, 1u);  // overflow: the caller fails the operation before writing
        return;
    }
    uint8_t* rec = arena + (uint64_t)slot * RECORD_BYTES;
    reinterpret_cast<uint32_t*>(rec)[0] = buf;
    reinterpret_cast<uint64_t*>(rec)[1] = e;
    const uint4* src = reinterpret_cast<const uint4*>(data + e * esize);
    uint4* dst = reinterpret_cast<uint4*>(rec + 16);
    for (uint32_t w = 0; w < esize / 16; ++w) dst[w] = src[w];
}

__global__ void k_restore(const uint8_t* __restrict__ arena, uint32_t count, uint8_t* const* __restrict__ bases,
                          const uint32_t* __restrict__ sizes) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= count) return;
    const uint8_t* rec = arena + (uint64_t)r * RECORD_BYTES;
    const uint32_t buf = reinterpret_cast<const uint32_t*>(rec)[0];
    const uint64_t e = reinterpret_cast<const uint64_t*>(rec)[1];
    const uint32_t esize = sizes[buf];
    const uint4* src = reinterpret_cast<const uint4*>(rec + 16);
    uint4* dst = reinterpret_cast<uint4*>(bases[buf] + e * esize);
    for (uint32_t w = 0; w < esize / 16; ++w) dst[w] = src[w];
}

__global__ void k_check_fr(const uint8_t* __restrict__ in, uint64_t n, uint32_t* __restrict__ bad) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t w[8];
    load_words(in + 32 * i, w);
    if (!Fr::is_canonical(w)) atomicMin(bad, (uint32_t)i);
}

__global__ void k_aff_to_xyzz(const G1A* __restrict__ in, uint64_t n, XYZZ<Fq>* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = XYZZ<Fq>::from_affine(in[i]);
}

// Canonical affine bytes of XYZZ (kind G1) or Montgomery affine (bases).
__global__ void k_to_wire(const uint8_t* __restrict__ src, uint32_t kind, uint64_t n, uint8_t* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    G1A a;
    if (kind == KIND_G1) a = reinterpret_cast<const XYZZ<Fq>*>(src)[i].to_affine();
    else a = reinterpret_cast<const G1A*>(src)[i];
    uint8_t* o = out + 64 * i;
    if (a.is_inf()) {
        const uint4 z = make_uint4(0, 0, 0, 0);
        for (int b = 0; b < 64; b += 16) *reinterpret_cast<uint4*>(o + b) = z;
        return;
    }
    store_canonical(o, a.x);
    store_canonical(o + 32, a.y);
}

__global__ void k_xyzz_to_affine(const XYZZ<Fq>* __restrict__ in, uint64_t n, G1A* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = in[i].to_affine();
}

__global__ void k_reverse(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst, uint64_t n, uint32_t esize) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint4* s = reinterpret_cast<const uint4*>(src + (n - 1 - i) * esize);
    uint4* d = reinterpret_cast<uint4*>(dst + i * esize);
    for (uint32_t w = 0; w < esize / 16; ++w) d[w] = s[w];
}

// [k] p, k canonical (left to right double-and-add).
DV_INL XYZZ<Fq> smul(const XYZZ<Fq>& p, const uint32_t* k) {
    int top = 255;
    while (top >= 0 && !((k[top >> 5] >> (top & 31)) & 1)) --top;
    if (top < 0 || p.is_inf()) return XYZZ<Fq>::inf();
    XYZZ<Fq> r = p;
    for (int i = top - 1; i >= 0; --i) {
        r = XYZZ<Fq>::dbl_paired(r);
        if ((k[i >> 5] >> (i & 31)) & 1) r = XYZZ<Fq>::add_paired(r, p);
    }
    return r;
}

// root^e (Montgomery) for a 64-bit exponent.
DV_INL Fr pow64(const Fr& root, uint64_t e) {
    Fr r = Fr::one();
    for (int b = 63; b >= 0; --b) {
        r = Fr::sqr(r);
        if ((e >> b) & 1) r = Fr::mul(r, root);
    }
    return r;
}

__global__ void k_transpose(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst, uint32_t kind, uint64_t start,
                            uint64_t n, uint64_t rows, uint64_t cols, const uint32_t* __restrict__ root_canon) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const uint64_t i = start + t, row = i / cols, col = i % cols, target = col * rows + row;
    if (kind == KIND_FR) {
        Fr v;
        load_words(src + 32 * i, v.v);
        if (root_canon) {
            uint32_t c[8];
            for (int w = 0; w < 8; ++w) c[w] = root_canon[w];
            v = Fr::mul(v, pow64(Fr::from_canonical(c), row * col));  // canonical x Montgomery = canonical
        }
        store_words(dst + 32 * target, v.v);
    } else {
        XYZZ<Fq> p = reinterpret_cast<const XYZZ<Fq>*>(src)[i];
        if (root_canon) {
            uint32_t c[8];
            for (int w = 0; w < 8; ++w) c[w] = root_canon[w];
            uint32_t k[8];
            pow64(Fr::from_canonical(c), row * col).to_canonical(k);
            p = smul(p, k);
        }
        reinterpret_cast<XYZZ<Fq>*>(dst)[target] = p;
    }
}

__global__ void k_zip(const uint8_t* __restrict__ a, const uint8_t* __restrict__ b, uint8_t* __restrict__ c, uint64_t n,
                      uint32_t op) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Fr x, y, r;
    load_words(a + 32 * i, x.v);
    load_words(b + 32 * i, y.v);
    if (op == 0) r = Fr::add(x, y);
    else if (op == 1) r = Fr::sub(x, y);
    else r = Fr::mul(Fr::mul(x, Fr::r2()), y);  // (x R) y R^-1 = x y
    store_words(c + 32 * i, r.v);
}

__global__ void __launch_bounds__(128) k_scale(const XYZZ<Fq>* __restrict__ pts, const uint8_t* __restrict__ sc,
                                               XYZZ<Fq>* __restrict__ out, uint64_t n) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t k[8];
    load_words(sc + 32 * i, k);
    out[i] = smul(pts[i], k);
}

inline unsigned grid_for(uint64_t n, unsigned t = 128) { return (unsigned)((n + t - 1) / t); }

// Canonical Fr check on 32 little-endian bytes (value < r).
bool fr_canonical_host(const uint8_t* b) {
    static const uint64_t R[4] = {0x43e1f593f0000001ull, 0x2833e84879b97091ull, 0xb85045b68181585dull,
                                  0x30644e72e131a029ull};
    uint64_t w[4];
    memcpy(w, b, 32);
    for (int i = 3; i >= 0; --i) {
        if (w[i] < R[i]) return true;
        if (w[i] > R[i]) return false;
    }
    return false;
}

// ----------------------------------------------------------------- state
struct ResBuffer {
    uint32_t kind = 0;
    uint64_t len = 0;
    bool writable = false;
    DevBuf data, marks;
};

uint64_t next_owner_tag() {
    static uint64_t tag = 0;
    return __atomic_add_fetch(&tag, 1, __ATOMIC_RELAXED);
}

}  // namespace

struct ResidentState {
    bool configured = false, sealed = false, in_tx = false;
    uint64_t owner = 0, limit = 0, journal_bytes = 0, allocated_device = 0;
    uint32_t epoch = 1, capacity = 0;
    std::vector<std::unique_ptr<ResBuffer>> buffers;
    DevBuf arena, ctl, temp, temp2, table;
    DvgpuResidentStats stats{};
    DvgpuResidentDiagnostics diag{};
};

namespace {

ResidentState& state_of(Backend& b) {
    if (!b.resident) throw InvalidArgument("resident backend is not configured");
    return *b.resident;
}

ResBuffer& buffer_of(ResidentState& s, uint64_t handle, uint32_t& index) {
    if ((handle >> 32) != s.owner) throw InvalidArgument("buffer belongs to another owner or is unknown");
    index = (uint32_t)(handle & 0xffffffffu);
    if (index >= s.buffers.size()) throw InvalidArgument("unknown buffer handle");
    return *s.buffers[index];
}

// validate(): kind, range, write permission (operators.rs:162-172).
ResBuffer& checked(ResidentState& s, uint64_t handle, uint32_t kind, uint64_t offset, uint64_t len, bool write,
                   uint32_t& index) {
    ResBuffer& buf = buffer_of(s, handle, index);
    if (buf.kind != kind) throw InvalidArgument(buf.kind == KIND_BASES ? "registered bases accept only READ and MSM_G1"
                                                                       : "buffer kind mismatch");
    if (offset + len < offset || offset + len > buf.len) throw InvalidArgument("buffer range out of bounds");
    if (write && s.sealed && !buf.writable) throw InvalidArgument("buffer is sealed read-only");
    return buf;
}

// validate_alias(): same buffer ranges may not overlap unless allowed exactly.
void check_alias(uint64_t src, uint64_t src_off, uint64_t dst, uint64_t dst_off, uint64_t len, bool exact_ok) {
    if (src != dst || len == 0) return;
    const bool overlaps = src_off < dst_off + len && dst_off < src_off + len;
    if (overlaps && !(exact_ok && src_off == dst_off)) throw InvalidArgument("overlapping buffer alias");
}

// Saves first-written elements of a destination range before the write.
void journal(Backend& b, ResidentState& s, ResBuffer& buf, uint32_t index, uint64_t offset, uint64_t n,
             uint64_t rows = 0, uint64_t cols = 0, bool transpose = false) {
    if (!s.in_tx || !n) return;
    uint32_t* ctl = s.ctl.view<uint32_t>();
    k_journal<<<grid_for(n, 256), 256, 0, b.stream>>>(buf.data.view<uint8_t>(), buf.marks.view<uint32_t>(),
                                                      elem_bytes(buf.kind), index, offset, n, rows, cols, transpose ? 1 : 0,
                                                      s.epoch, s.arena.view<uint8_t>(), s.capacity, ctl);
    DV_LAUNCH();
    uint32_t h[2] = {0, 0};
    DV_CUDA(cudaMemcpyAsync(h, ctl, sizeof h, cudaMemcpyDeviceToHost, b.stream));
    DV_CUDA(cudaStreamSynchronize(b.stream));
    if (h[1]) throw InvalidArgument("resident transaction exceeds the journal arena");
    const uint64_t saved = std::min<uint64_t>(h[0], s.capacity);
    s.diag.journal_saved_ranges++;
    s.diag.journal_saved_bytes = saved * elem_bytes(buf.kind);
    s.diag.journal_peak_bytes = std::max<uint64_t>(s.diag.journal_peak_bytes, saved * RECORD_BYTES);
}

uint8_t* at(ResBuffer& buf, uint64_t e) { return buf.data.view<uint8_t>() + e * elem_bytes(buf.kind); }

// One resident operation (dvgpu_resident_call).
uint64_t resident_op(Backend& b, const DvgpuResidentOp& op) {
    ResidentState& s = state_of(b);
    const cudaStream_t st = b.stream;
    uint32_t ia = 0, ib = 0, ic = 0;
    switch (op.opcode) {
    case OP_LENGTH: return buffer_of(s, op.a, ia).len;
    case OP_KIND: return buffer_of(s, op.a, ia).kind;
    case OP_BEGIN:
        if (s.in_tx) throw InvalidArgument("transaction already active");
        s.in_tx = true;
        s.epoch++;
        DV_CUDA(cudaMemsetAsync(s.ctl.view<uint32_t>(), 0, 2 * sizeof(uint32_t), st));
        s.stats.calls++;
        return 0;
    case OP_ROLLBACK: {
        if (!s.in_tx) throw InvalidArgument("no transaction to roll back");
        uint32_t count = 0;
        DV_CUDA(cudaMemcpyAsync(&count, s.ctl.view<uint32_t>(), 4, cudaMemcpyDeviceToHost, st));
        DV_CUDA(cudaStreamSynchronize(st));
        count = std::min(count, s.capacity);
        if (count) {
            const size_t nb = s.buffers.size();
            std::vector<uint8_t*> ptrs(nb);
            std::vector<uint32_t> sizes(nb);
            for (size_t k = 0; k < nb; ++k) {
                ptrs[k] = s.buffers[k]->data.view<uint8_t>();
                sizes[k] = elem_bytes(s.buffers[k]->kind);
            }
            uint8_t* t = s.table.as<uint8_t>(nb * (sizeof(void*) + 4));
            DV_CUDA(cudaMemcpyAsync(t, ptrs.data(), nb * sizeof(void*), cudaMemcpyHostToDevice, st));
            DV_CUDA(cudaMemcpyAsync(t + nb * sizeof(void*), sizes.data(), nb * 4, cudaMemcpyHostToDevice, st));
            k_restore<<<grid_for(count, 256), 256, 0, st>>>(s.arena.view<uint8_t>(), count,
                                                            reinterpret_cast<uint8_t* const*>(t),
                                                            reinterpret_cast<const uint32_t*>(t + nb * sizeof(void*)));
            DV_LAUNCH();
            DV_CUDA(cudaStreamSynchronize(st));
        }
        s.in_tx = false;
        s.epoch++;  // every marker of the rolled-back transaction is stale now
        s.stats.calls++;
        return 0;
    }
    case OP_ALLOC:
    case OP_ALLOC_BASES: {
        const bool packed = op.opcode == OP_ALLOC_BASES;
        if (s.sealed) throw InvalidArgument("resident allocation after seal");
        if (s.in_tx) throw InvalidArgument("buffer allocation in transaction");
        const uint32_t kind = packed ? KIND_BASES : op.kind;
        if (kind > KIND_G1 && !packed) throw InvalidArgument("unknown buffer kind");
        if (packed && op.length && !op.input) throw InvalidArgument("null basis input");
        const uint64_t bytes = op.length * (elem_bytes(kind) + (packed ? 0 : 4));
        if (s.allocated_device + bytes > s.limit) throw InvalidArgument("resident allocation exceeds the memory limit");
        auto buf = std::make_unique<ResBuffer>();
        buf->kind = kind;
        buf->len = op.length;
        buf->writable = !packed && (op.flags & 1);
        uint8_t* d = buf->data.as<uint8_t>(std::max<uint64_t>(1, op.length) * elem_bytes(kind));
        if (!packed) {
            DV_CUDA(cudaMemsetAsync(d, 0, op.length * elem_bytes(kind), st));  // zero / infinity
            uint32_t* m = buf->marks.as<uint32_t>(std::max<uint64_t>(1, op.length));
            DV_CUDA(cudaMemsetAsync(m, 0, op.length * 4, st));
        } else if (op.length) {
            uint8_t* wire = s.temp.as<uint8_t>(op.length * 64);
            DV_CUDA(cudaMemcpyAsync(wire, op.input, op.length * 64, cudaMemcpyHostToDevice, st));
            uint32_t* bad = b.err.as<uint32_t>(1);
            DV_CUDA(cudaMemsetAsync(bad, 0xff, 4, st));
            convert_points<Fq>(wire, reinterpret_cast<G1A*>(d), op.length, bad, st);
            if (read_err_word(b, bad, st) != 0xffffffffu) throw InvalidArgument("invalid G1 basis");
            s.stats.h2d_bytes += op.length * 64;
        }
        DV_CUDA(cudaStreamSynchronize(st));
        s.allocated_device += bytes;
        s.stats.bytes_allocated += op.length * (kind == KIND_FR ? 32 : 64);
        s.diag.resident_allocations++;
        s.stats.calls++;
        s.buffers.push_back(std::move(buf));
        return (s.owner << 32) | (uint64_t)(s.buffers.size() - 1);
    }
    case OP_WRITE: {
        if (op.kind > KIND_G1) throw InvalidArgument("WRITE takes Fr or G1 buffers");
        ResBuffer& dst = checked(s, op.a, op.kind, op.a_offset, op.length, true, ia);
        if (op.length && !op.input) throw InvalidArgument("null write input");
        if (!op.length) { s.stats.calls++; return 0; }
        uint32_t* bad = b.err.as<uint32_t>(1);
        DV_CUDA(cudaMemsetAsync(bad, 0xff, 4, st));
        if (op.kind == KIND_FR) {
            uint8_t* staged = s.temp.as<uint8_t>(op.length * 32);
            DV_CUDA(cudaMemcpyAsync(staged, op.input, op.length * 32, cudaMemcpyHostToDevice, st));
            k_check_fr<<<grid_for(op.length), 128, 0, st>>>(staged, op.length, bad);
            DV_LAUNCH();
            if (read_err_word(b, bad, st) != 0xffffffffu) throw InvalidArgument("non-canonical Fr value");
            journal(b, s, dst, ia, op.a_offset, op.length);
            DV_CUDA(cudaMemcpyAsync(at(dst, op.a_offset), staged, op.length * 32, cudaMemcpyDeviceToDevice, st));
            s.stats.h2d_bytes += op.length * 32;
        } else {
            uint8_t* wire = s.temp.as<uint8_t>(op.length * 64);
            G1A* aff = s.temp2.as<G1A>(op.length);
            DV_CUDA(cudaMemcpyAsync(wire, op.input, op.length * 64, cudaMemcpyHostToDevice, st));
            convert_points<Fq>(wire, aff, op.length, bad, st);
            if (read_err_word(b, bad, st) != 0xffffffffu) throw InvalidArgument("invalid resident G1 point");
            journal(b, s, dst, ia, op.a_offset, op.length);
            k_aff_to_xyzz<<<grid_for(op.length), 128, 0, st>>>(aff, op.length,
                                                              reinterpret_cast<XYZZ<Fq>*>(at(dst, op.a_offset)));
            DV_LAUNCH();
            s.stats.h2d_bytes += op.length * 64;
        }
        DV_CUDA(cudaStreamSynchronize(st));
        s.stats.calls++;
        return 0;
    }
    case OP_READ: {
        ResBuffer& src = buffer_of(s, op.a, ia);
        const uint32_t kind = src.kind == KIND_BASES ? KIND_G1 : src.kind;
        if (op.kind != kind) throw InvalidArgument("buffer kind mismatch");
        if ((kind == KIND_FR && op.flags) || op.flags > 1) throw InvalidArgument("unsupported READ flags");
        if (op.a_offset + op.length > src.len) throw InvalidArgument("buffer range out of bounds");
        if (op.length && !op.output) throw InvalidArgument("null read output");
        if (op.length) {
            if (kind == KIND_FR) {
                DV_CUDA(cudaMemcpyAsync(op.output, at(src, op.a_offset), op.length * 32, cudaMemcpyDeviceToHost, st));
                s.stats.d2h_bytes += op.length * 32;
            } else {
                uint8_t* wire = s.temp.as<uint8_t>(op.length * 64);
                k_to_wire<<<grid_for(op.length), 128, 0, st>>>(at(src, op.a_offset), src.kind, op.length, wire);
                DV_LAUNCH();
                DV_CUDA(cudaMemcpyAsync(op.output, wire, op.length * 64, cudaMemcpyDeviceToHost, st));
                s.stats.d2h_bytes += op.length * 64;
            }
            DV_CUDA(cudaStreamSynchronize(st));
        }
        s.stats.calls++;
        return 0;
    }
    case OP_COPY:
    case OP_REVERSE: {
        const bool rev = op.opcode == OP_REVERSE;
        const uint32_t kind = rev ? op.kind : buffer_of(s, op.a, ia).kind;
        if (kind > KIND_G1) throw InvalidArgument("registered bases accept only READ and MSM_G1");
        ResBuffer& src = checked(s, op.a, kind, op.a_offset, op.length, false, ia);
        ResBuffer& dst = checked(s, op.c, kind, op.c_offset, op.length, true, ic);
        check_alias(op.a, op.a_offset, op.c, op.c_offset, op.length, rev ? op.length <= 1 : true);
        if (op.length && !(op.a == op.c && op.a_offset == op.c_offset)) {
            journal(b, s, dst, ic, op.c_offset, op.length);
            if (rev) {
                k_reverse<<<grid_for(op.length), 128, 0, st>>>(at(src, op.a_offset), at(dst, op.c_offset), op.length,
                                                               elem_bytes(kind));
                DV_LAUNCH();
            } else {
                DV_CUDA(cudaMemcpyAsync(at(dst, op.c_offset), at(src, op.a_offset), op.length * elem_bytes(kind),
                                        cudaMemcpyDeviceToDevice, st));
            }
            DV_CUDA(cudaStreamSynchronize(st));
            s.diag.explicit_d2d_bytes += op.length * elem_bytes(kind);
        }
        s.stats.calls++;
        return 0;
    }
    case OP_TRANSPOSE: {
        if (op.kind > KIND_G1) throw InvalidArgument("registered bases accept only READ and MSM_G1");
        if (!op.rows || !op.cols) throw InvalidArgument("transpose dimensions must be positive");
        const uint64_t size = op.rows * op.cols;
        if (op.cols && size / op.cols != op.rows) throw InvalidArgument("transpose size overflow");
        if (op.a_offset + op.length > size) throw InvalidArgument("transpose range out of bounds");
        ResBuffer& src = checked(s, op.a, op.kind, 0, size, false, ia);
        ResBuffer& dst = checked(s, op.c, op.kind, 0, size, true, ic);
        if (op.a == op.c && op.length) throw InvalidArgument("transpose requires distinct buffers");
        if ((op.flags & 1) && !op.input) throw InvalidArgument("null transpose root");
        if (op.length) {
            uint32_t* root = nullptr;
            if (op.flags & 1) {
                if (!fr_canonical_host(op.input)) throw InvalidArgument("non-canonical transpose root");
                root = s.temp.as<uint32_t>(8);
                DV_CUDA(cudaMemcpyAsync(root, op.input, 32, cudaMemcpyHostToDevice, st));
            }
            journal(b, s, dst, ic, op.a_offset, op.length, op.rows, op.cols, true);
            k_transpose<<<grid_for(op.length), 128, 0, st>>>(src.data.view<uint8_t>(), dst.data.view<uint8_t>(),
                                                            op.kind, op.a_offset, op.length, op.rows, op.cols, root);
            DV_LAUNCH();
            DV_CUDA(cudaStreamSynchronize(st));
        }
        s.stats.calls++;
        return 0;
    }
    case OP_TRANSFORM:
    case OP_TRANSFORM_PACKET: {
        const bool packet = op.opcode == OP_TRANSFORM_PACKET;
        if (op.kind > KIND_G1) throw InvalidArgument("registered bases accept only READ and MSM_G1");
        const uint64_t row_len = packet ? op.length : op.cols;
        const uint64_t rows = packet ? 1 : op.rows;
        const uint64_t first = packet ? 0 : op.a_offset;
        int logn = 0;
        while ((1ull << logn) < row_len) ++logn;
        if (!row_len || (1ull << logn) != row_len || logn > 20)
            throw InvalidArgument("transform row length must be a power of two up to 2^20");
        if (packet && row_len > MAX_PACKET) throw InvalidArgument("transform packet length outside 1..4096");
        const uint64_t start = first * row_len, count = rows * row_len;
        ResBuffer& src = checked(s, op.a, op.kind, start, count, false, ia);
        ResBuffer& dst = checked(s, op.c, op.kind, start, count, true, ic);
        if (packet) {
            ResBuffer& scratch = checked(s, op.b, op.kind, 0, count, true, ib);
            (void)scratch;
            if (op.a == op.b || op.b == op.c) throw InvalidArgument("transform packet requires distinct buffers");
        }
        if (op.a == op.c && count) throw InvalidArgument("row transform requires distinct buffers");
        if (count) {
            journal(b, s, dst, ic, start, count);
            const bool inverse = op.flags & 1;
            if (op.kind == KIND_FR) {
                std::vector<NttBatchItem> items;
                for (uint64_t r = 0; r < rows; ++r)
                    items.push_back(NttBatchItem{at(src, start + r * row_len), at(dst, start + r * row_len), logn,
                                                 inverse ? NTT_INVERSE : NTT_FORWARD});
                if (logn == 0) {
                    DV_CUDA(cudaMemcpyAsync(at(dst, start), at(src, start), count * 32, cudaMemcpyDeviceToDevice, st));
                } else {
                    NttBatch batch;
                    ntt_batch_prepare(b.ntt, batch, items, st);
                    ntt_batch_enqueue(batch, st);
                    ntt_batch_check(batch, st);
                }
                s.stats.fr_transform_elements += count;
            } else {
                XYZZ<Fq>* work = s.temp2.as<XYZZ<Fq>>(count);
                DV_CUDA(cudaMemcpyAsync(work, at(src, start), count * 128, cudaMemcpyDeviceToDevice, st));
                g1_ntt_rows_xyzz(b.ntt, work, logn, rows, inverse, reinterpret_cast<XYZZ<Fq>*>(at(dst, start)), st);
                s.stats.g1_transform_elements += count;
            }
            DV_CUDA(cudaStreamSynchronize(st));
        }
        s.stats.calls++;
        return 0;
    }
    case OP_ZIP: {
        if (op.flags > 2) throw InvalidArgument("unknown field operation");
        ResBuffer& l = checked(s, op.a, KIND_FR, op.a_offset, op.length, false, ia);
        ResBuffer& r = checked(s, op.b, KIND_FR, op.b_offset, op.length, false, ib);
        ResBuffer& d = checked(s, op.c, KIND_FR, op.c_offset, op.length, true, ic);
        check_alias(op.a, op.a_offset, op.c, op.c_offset, op.length, true);
        check_alias(op.b, op.b_offset, op.c, op.c_offset, op.length, true);
        if (op.length) {
            journal(b, s, d, ic, op.c_offset, op.length);
            k_zip<<<grid_for(op.length), 128, 0, st>>>(at(l, op.a_offset), at(r, op.b_offset), at(d, op.c_offset),
                                                       op.length, op.flags);
            DV_LAUNCH();
            DV_CUDA(cudaStreamSynchronize(st));
        }
        s.stats.calls++;
        return 0;
    }
    case OP_SCALE: {
        ResBuffer& p = checked(s, op.a, KIND_G1, op.a_offset, op.length, false, ia);
        ResBuffer& f = checked(s, op.b, KIND_FR, op.b_offset, op.length, false, ib);
        ResBuffer& d = checked(s, op.c, KIND_G1, op.c_offset, op.length, true, ic);
        check_alias(op.a, op.a_offset, op.c, op.c_offset, op.length, true);
        if (op.length) {
            journal(b, s, d, ic, op.c_offset, op.length);
            k_scale<<<grid_for(op.length), 128, 0, st>>>(reinterpret_cast<const XYZZ<Fq>*>(at(p, op.a_offset)),
                                                         at(f, op.b_offset),
                                                         reinterpret_cast<XYZZ<Fq>*>(at(d, op.c_offset)), op.length);
            DV_LAUNCH();
            DV_CUDA(cudaStreamSynchronize(st));
        }
        s.stats.calls++;
        return 0;
    }
    case OP_MSM_G1: {
        ResBuffer& p = buffer_of(s, op.a, ia);
        if (p.kind == KIND_FR) throw InvalidArgument("buffer kind mismatch");
        if (op.a_offset + op.length > p.len) throw InvalidArgument("buffer range out of bounds");
        ResBuffer& f = checked(s, op.b, KIND_FR, op.b_offset, op.length, false, ib);
        if (!op.output) throw InvalidArgument("null MSM output");
        if (!op.length) {
            memset(op.output, 0, 64);
        } else {
            const G1A* pts;
            if (p.kind == KIND_BASES) {
                pts = reinterpret_cast<const G1A*>(at(p, op.a_offset));
            } else {
                G1A* aff = s.temp2.as<G1A>(op.length);
                k_xyzz_to_affine<<<grid_for(op.length), 128, 0, st>>>(
                    reinterpret_cast<const XYZZ<Fq>*>(at(p, op.a_offset)), op.length, aff);
                DV_LAUNCH();
                pts = aff;
            }
            const std::vector<uint32_t> offs = {0u, (uint32_t)op.length};
            uint8_t out[64];
            msm_run<Fq>(b.msm, pts, reinterpret_cast<const uint32_t*>(at(f, op.b_offset)), offs.data(), 1, 0, st,
                        out, &b.msm_stats);
            memcpy(op.output, out, 64);
        }
        s.stats.msm_g1_points += op.length;
        s.stats.d2h_bytes += 64;
        s.stats.calls++;
        return 0;
    }
    case OP_MSM_G2: {
        ResBuffer& f = checked(s, op.b, KIND_FR, op.b_offset, op.length, false, ib);
        if (!op.output || (op.length && !op.input)) throw InvalidArgument("invalid G2 MSM buffers");
        if (!op.length) {
            memset(op.output, 0, 128);
        } else {
            uint8_t* wire = s.temp.as<uint8_t>(op.length * 128);
            G2A* aff = reinterpret_cast<G2A*>(s.temp2.as<uint8_t>(op.length * sizeof(G2A)));
            DV_CUDA(cudaMemcpyAsync(wire, op.input, op.length * 128, cudaMemcpyHostToDevice, st));
            uint32_t* bad = b.err.as<uint32_t>(1);
            DV_CUDA(cudaMemsetAsync(bad, 0xff, 4, st));
            convert_points<Fq2>(wire, aff, op.length, bad, st);
            if (read_err_word(b, bad, st) != 0xffffffffu) throw InvalidArgument("invalid resident G2 base");
            const std::vector<uint32_t> offs = {0u, (uint32_t)op.length};
            uint8_t out[128];
            msm_run<Fq2>(b.msm, aff, reinterpret_cast<const uint32_t*>(at(f, op.b_offset)), offs.data(), 1, 0, st,
                         out, &b.msm_stats);
            memcpy(op.output, out, 128);
        }
        s.stats.msm_g2_points += op.length;
        s.stats.h2d_bytes += op.length * 128;
        s.stats.d2h_bytes += 128;
        s.stats.calls++;
        return 0;
    }
    default:
        throw InvalidArgument("unknown resident opcode");
    }
}

}  // namespace
}  // namespace dv

using namespace dv;

extern "C" int dvgpu_resident_configure(void* opaque, uint64_t memory_limit_bytes, uint64_t journal_bytes,
                                        const uint8_t* root, char* error, size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) {
        require(!b.resident, "resident backend already configured");
        require(root && root_order_2_20(root), "resident root must have multiplicative order exactly 2^20");
        require(journal_bytes >= RECORD_BYTES && journal_bytes <= memory_limit_bytes,
                "journal arena must hold at least one record and fit the memory limit");
        auto s = std::make_unique<ResidentState>();
        s->owner = next_owner_tag();
        s->limit = memory_limit_bytes;
        s->journal_bytes = journal_bytes;
        s->capacity = (uint32_t)std::min<uint64_t>(journal_bytes / RECORD_BYTES, 0xffffffffu);
        s->arena.as<uint8_t>((uint64_t)s->capacity * RECORD_BYTES);
        s->ctl.as<uint32_t>(2);
        DV_CUDA(cudaMemsetAsync(s->ctl.view<uint32_t>(), 0, 8, b.stream));
        DV_CUDA(cudaStreamSynchronize(b.stream));
        s->allocated_device = journal_bytes;
        s->diag.journal_metadata_capacity_bytes = (uint64_t)s->capacity * 16;
        s->configured = true;
        b.resident = std::move(s);
    });
}

extern "C" int dvgpu_resident_call(void* opaque, const DvgpuResidentOp* operation, uint64_t* result, char* error,
                                   size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) {
        require(operation != nullptr, "null resident operation");
        const uint64_t r = resident_op(b, *operation);
        if (result) *result = r;
        b.resident->diag.device_operations++;
    });
}

extern "C" void dvgpu_resident_seal(void* opaque) {
    auto* b = static_cast<Backend*>(opaque);
    if (b && b->resident) b->resident->sealed = true;
}

extern "C" void dvgpu_resident_commit(void* opaque) {
    auto* b = static_cast<Backend*>(opaque);
    if (!b || !b->resident || !b->resident->in_tx) return;
    // host metadata only: the next transaction's epoch makes every marker stale
    b->resident->in_tx = false;
    b->resident->epoch++;
    b->resident->stats.calls++;
}

extern "C" int dvgpu_resident_stats(void* opaque, DvgpuResidentStats* out) {
    auto* b = static_cast<Backend*>(opaque);
    if (!b || !out) return -1;
    *out = b->resident ? b->resident->stats : DvgpuResidentStats{};
    return 0;
}

extern "C" int dvgpu_resident_diagnostics(void* opaque, DvgpuResidentDiagnostics* out) {
    auto* b = static_cast<Backend*>(opaque);
    if (!b || !out) return -1;
    *out = b->resident ? b->resident->diag : DvgpuResidentDiagnostics{};
    return 0;
}
