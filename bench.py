#!/usr/bin/env python
"""Benchmark of the BN254 prover hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--op msm] [--log-n 20] [--impl ours|reference]

Default (the headline): G1 MSM over 2^20 points, bases [tau^i]G1 (seeded
tau), uniform Fr scalars.  Other operators of the same path: --op g2msm,
ntt (--kind forward|inverse|coset_forward|coset_inverse), sparse (--k, over
2^16 resident bases), fixedbase.  One JSON line on stdout (rank 0).

A step is one complete operator call on device-resident inputs; its result
is a canonical value in host memory (MSM: affine point; NTT: the device
output vector).

  value / ms_per_step : device time per step (CUDA events on the launching
                        stream), L2 flushed (256 MB write) between steps, the
                        sum over K steps / K.  With N GPUs the ranks run
                        independent replicas (nothing is sharded);
                        value = max-over-ranks time / (N * K).
  e2e                 : the same operator through the reference-facing C-ABI
                        call with pinned HOST buffers (host->device input
                        copies and the result copy inside the timed region).
  roofline            : integer-multiply bound.  MSM: the bucket-accumulation
                        kernel, (points x windows) XYZZ mixed additions x (8
                        Fq products x 136 + 2 Fq squares x 108) 32x32->64-bit
                        multiply-accumulates per launch, over its CUDA-event
                        duration.  Other operators: the whole call, with the
                        algorithmic multiplication count stated in the line.
                        Peak = IMAD rate measured in this run.
  cpu_baseline        : the CPU oracle (C++ restatement of arkworks
                        semantics) on the same inputs, all host threads.
  --op poly           : the polynomial field work of one sparse update over
                        2^log-n affected points (host-buffer entry points;
                        value = e2e).
  --impl reference    : that CPU implementation alone, on the same workload
                        (the reference's Rust + arkworks + ICICLE code cannot
                        be built in this image).
"""
import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NTT_KINDS = {"forward": 0, "inverse": 1, "coset_forward": 2, "coset_inverse": 3}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--op", default="proofs", choices=["msmres", "msm", "g2msm", "ntt", "sparse", "fixedbase", "batch", "g2check",
                                                         "serve", "ecntt", "poly", "pairing", "proofs"])
    ap.add_argument("--log-n", type=int, default=None)
    ap.add_argument("--kind", default="forward", choices=list(NTT_KINDS))
    ap.add_argument("--k", type=int, default=4096, help="sparse: entries per request")
    ap.add_argument("--alg", type=int, default=3, choices=[1, 2, 3], help="g2check: subgroup algorithm")
    ap.add_argument("--requests", type=int, default=None, help="serve / proofs: update requests per run")
    ap.add_argument("--sessions", type=int, default=64, help="proofs: sessions of n = 2^log-n")
    ap.add_argument("--mix", action="store_true", help="proofs: 64 sessions, n in {256, 4096, 65536}, 37:18:9")
    ap.add_argument("--umax", type=float, default=9.0,
                    help="proofs: floor(2^U) multiplication gates, U~U[0,umax] (2 witness indices each)")
    ap.add_argument("--rows", type=int, default=16, help="ecntt: rows per transform call")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--probe", choices=["update", "batch"], default=None,
                    help="proofs: run one fixed case for a profiler and exit (no timing line): 'update' = two "
                         "sessions of n = 2^log-n opened, then one per-call update of 64 gates; 'batch' = 64 "
                         "sessions, then one served batch of 64 updates")
    ap.add_argument("--no-operators", action="store_true",
                    help="proofs: leave out the MSM 2^20 / NTT 2^22 operator points")
    a = ap.parse_args()
    if a.log_n is None:
        a.log_n = {"msm": 20, "msmres": 20, "g2msm": 16, "ntt": 22, "sparse": 16, "fixedbase": 20, "batch": 18,
                   "g2check": 16, "serve": 16, "ecntt": 12, "poly": 12, "pairing": 12, "proofs": 16}[a.op]
    if a.requests is None:
        a.requests = {"serve": 4000, "proofs": 512}.get(a.op, 4000)
    if a.steps is None:
        a.steps = {"msm": 200, "msmres": 200, "g2msm": 50, "ntt": 200, "sparse": 200, "fixedbase": 100,
                   "batch": 20, "g2check": 50, "serve": 1, "proofs": 1,
                   "ecntt": 10, "poly": 20, "pairing": 20}[a.op]
    return a


# 32x32->64-bit multiply-accumulates of one Montgomery product and one
# Montgomery square (cross products once, then the reduction) over Fq.
MAC_MUL, MAC_SQR = 136, 108
# XYZZ mixed addition (madd-2008-s: 8 products, 2 squares) and full addition
# (add-2008-s: 12 products, 2 squares) over Fq; over Fq2 a product is three
# Fq products (Karatsuba) and a square two.
G1_MADD_MACS = 8 * MAC_MUL + 2 * MAC_SQR
G1_ADD_MACS = 12 * MAC_MUL + 2 * MAC_SQR
G2_MADD_MACS = (8 * 3 + 2 * 2) * MAC_MUL
G2_ADD_MACS = (12 * 3 + 2 * 2) * MAC_MUL


def msm_macs(n, g2=False):
    """Algorithmic work of an n-point MSM in multiply-accumulates: min over c
    of ceil(254/c) * (n mixed additions + 2^c full additions: two per bucket
    of the bucket reduction)."""
    if n <= 0:
        return 0
    madd, add = (G2_MADD_MACS, G2_ADD_MACS) if g2 else (G1_MADD_MACS, G1_ADD_MACS)
    return min(math.ceil(254 / c) * (madd * n + add * (1 << c)) for c in range(2, 24))


class ClockSampler:
    """nvidia-smi samples of one GPU during the timed region."""

    FIELDS = ("index,pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id):
        self.bus_id = (bus_id or "").lower()
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        rows = []
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 10:
                continue
            bus = parts[1].lower()
            if self.bus_id and not (bus.endswith(self.bus_id[-12:]) or self.bus_id.endswith(bus[-12:])):
                continue
            rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = sorted(v for v in (num(r[2]) for r in rows) if v is not None)
        mx = max(v for v in (num(r[3]) for r in rows) if v is not None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[6 + k].lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}


class _DeviceBytes:
    """A raw device pointer as a CUDA array (for torch.as_tensor)."""

    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False),
                                         "version": 3}


def device_view(torch, ptr, nbytes):
    return torch.as_tensor(_DeviceBytes(ptr, nbytes), device="cuda")


def load_traffic(name, key="traffic_bytes_per_launch"):
    """DRAM bytes of the dominant kernel from the committed ncu summary
    profiles/<name>.txt (line '<key>: X', per launch by default)."""
    path = os.path.join(ROOT, "profiles", name + ".txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith(key + ":"):
            try:
                return float(line.split(":", 1)[1])
            except ValueError:
                return None
    return None


# ----------------------------------------------------------------- operators
class MsmOp:
    def __init__(self, args, g2=False):
        self.g2 = g2
        self.n = 1 << args.log_n
        self.size = 128 if g2 else 64
        self.metric = f"{'G2' if g2 else 'G1'} MSM 2^{args.log_n} ms"
        self.workload = (f"{'G2' if g2 else 'G1'} MSM 2^{args.log_n}: bases [tau^i]{'G2' if g2 else 'G1'} affine "
                         f"(seeded tau), uniform Fr scalars")
        self.profile = f"msm_{'g2' if g2 else 'g1'}_accum_2p{args.log_n}"

    def setup(self, torch, b, s, rank):
        n = self.n
        tau = torch.empty(32, dtype=torch.uint8, device="cuda")
        b.random_fr_device(2812, 1, tau.data_ptr(), s)
        powers = torch.empty(n * 32, dtype=torch.uint8, device="cuda")
        b.fr_powers_device(tau.data_ptr(), n, powers.data_ptr(), s)
        self.points = torch.empty(n * self.size, dtype=torch.uint8, device="cuda")
        b.fixed_base_device(powers.data_ptr(), n, self.g2, self.points.data_ptr(), s)
        self.scalars = torch.empty(n * 32, dtype=torch.uint8, device="cuda")
        b.random_fr_device(2813 + rank, n, self.scalars.data_ptr(), s)
        torch.cuda.synchronize()
        self.tuned_c, self.tune_log = b.autotune_msm(n, g2=self.g2)
        self.config = {"points": n, "window_bits": self.tuned_c, "windows": math.ceil(255 / self.tuned_c)}

    def step(self, b, s):
        return b.msm_device(self.points.data_ptr(), self.scalars.data_ptr(), self.n, g2=self.g2, stream=s)

    def host_inputs(self, torch):
        self.h_points = torch.empty(self.n * self.size, dtype=torch.uint8, pin_memory=True)
        self.h_scalars = torch.empty(self.n * 32, dtype=torch.uint8, pin_memory=True)
        self.h_points.copy_(self.points)
        self.h_scalars.copy_(self.scalars)
        self.out = ctypes.create_string_buffer(self.size)

    def e2e_step(self, dv, b):
        fn = dv.lib().dvgpu_bn254_g2_msm if self.g2 else dv.lib().dvgpu_bn254_msm
        err = ctypes.create_string_buffer(256)
        rc = fn(b.handle, self.h_points.data_ptr(), self.h_scalars.data_ptr(), self.n, self.out, err, 256)
        if rc != 0:
            raise RuntimeError(err.value)
        return self.out.raw

    def e2e_bytes(self):
        return self.n * (self.size + 32), self.size + self.config["windows"] * 2 * self.size

    def roofline(self, tl, imad_peak, step_ms):
        macs_total = msm_macs(self.n, self.g2)
        accum_ms = tl.ms[3] / max(1, tl.calls)
        adds = tl.accum_mixed_adds / max(1, tl.calls)
        macs = adds * (G2_MADD_MACS if self.g2 else G1_MADD_MACS)
        ach = macs / (accum_ms * 1e-3) / 1e12
        return ({"bound": "imad", "kernel": "k_accum (bucket accumulation)", "achieved": ach,
                 "peak": imad_peak / 1e12, "unit": "TMAC/s", "frac": ach / (imad_peak / 1e12),
                 "algorithmic_macs_per_launch": macs, "launch_ms": accum_ms},
                {"algorithmic_macs": macs_total, "achieved_tmacs": macs_total / (step_ms * 1e-3) / 1e12,
                 "frac": macs_total / (step_ms * 1e-3) / imad_peak})

    def cpu(self, oracle, threads):
        pts = bytes(self.h_points.numpy().tobytes())
        sc = bytes(self.h_scalars.numpy().tobytes())
        t0 = time.perf_counter()
        out = (oracle.msm_g2 if self.g2 else oracle.msm_g1)(pts, sc, threads=threads)
        return out, (time.perf_counter() - t0) * 1e3, f"one full 2^{int(math.log2(self.n))}-point MSM on the same inputs"


class ResidentMsmOp(MsmOp):
    """G1 MSM over a registered (HBM-resident) SRS with precomputed window
    multiples (dvgpu_bases_precompute, setup, not timed): every window adds
    into one shared bucket set.  e2e stays the reference-facing per-call
    dvgpu_bn254_msm with host buffers."""

    def __init__(self, args):
        super().__init__(args, g2=False)
        self.workload = (self.workload + "; SRS resident in HBM with precomputed window multiples "
                         "(registration and precomputation are setup, not timed)")
        self.profile = f"msm_g1_resident_accum_2p{args.log_n}"

    def setup(self, torch, b, s, rank):
        super().setup(torch, b, s, rank)
        torch.cuda.synchronize()
        self.handle = b.register_bases(self.points.cpu().numpy().tobytes())
        self.pre_c = b.precompute_bases(self.handle, 0)
        self.config = {"points": self.n, "window_bits": self.pre_c, "windows": math.ceil(255 / self.pre_c),
                       "precomputed_table_bytes": self.n * math.ceil(255 / self.pre_c) * 64}
        self.tune_log = None

    def step(self, b, s):
        return b.msm_resident(self.handle, self.scalars.data_ptr(), self.n, stream=s)

    def e2e_step(self, dv, b):
        # the per-request call of a resident prover: scalars from host memory
        err = ctypes.create_string_buffer(256)
        rc = dv.lib().dvgpu_bn254_msm_resident_host(b.handle, self.handle, self.h_scalars.data_ptr(), self.n,
                                                    self.out, err, 256)
        if rc != 0:
            raise RuntimeError(err.value)
        return self.out.raw

    def e2e_bytes(self):
        return self.n * 32, 64


class NttOp:
    def __init__(self, args):
        self.n = 1 << args.log_n
        self.logn = args.log_n
        self.kind = NTT_KINDS[args.kind]
        self.kind_name = args.kind
        self.metric = f"Fr NTT 2^{args.log_n} ms ({args.kind})"
        self.workload = f"Fr radix-2 NTT 2^{args.log_n} {args.kind} (arkworks domain, coset g=5) on uniform Fr"
        self.profile = f"ntt_pass_2p{args.log_n}"

    def setup(self, torch, b, s, rank):
        self.src = torch.empty(self.n * 32, dtype=torch.uint8, device="cuda")
        b.random_fr_device(3000 + rank, self.n, self.src.data_ptr(), s)
        self.dst = torch.empty_like(self.src)
        torch.cuda.synchronize()
        self.tune_log = None
        self.config = {"elements": self.n, "kind": self.kind_name, "passes": (self.logn + 10) // 11}

    def step(self, b, s):
        b.ntt_device(self.src.data_ptr(), self.n, self.kind, self.dst.data_ptr(), s)
        return None

    def host_inputs(self, torch):
        self.h_src = torch.empty(self.n * 32, dtype=torch.uint8, pin_memory=True)
        self.h_src.copy_(self.src)
        self.h_dst = torch.empty(self.n * 32, dtype=torch.uint8, pin_memory=True)

    def e2e_step(self, dv, b):
        err = ctypes.create_string_buffer(256)
        dst = ctypes.cast(ctypes.c_void_p(self.h_dst.data_ptr()), ctypes.c_char_p)
        rc = dv.lib().dvgpu_bn254_ntt_ex(b.handle, self.h_src.data_ptr(), self.n, self.kind, dst, err, 256)
        if rc != 0:
            raise RuntimeError(err.value)
        return None

    def e2e_bytes(self):
        return self.n * 32, self.n * 32

    def fme(self):
        extra = self.n if self.kind in (1, 2) else (2 * self.n if self.kind == 3 else 0)
        return self.n // 2 * self.logn + extra

    def roofline(self, tl, imad_peak, step_ms):
        macs = self.fme() * 136
        ach = macs / (step_ms * 1e-3) / 1e12
        hbm = 64 * self.n / (step_ms * 1e-3) / 1e9
        r = {"bound": "imad", "kernel": "whole NTT (k_dif_pass passes + k_permute)", "achieved": ach,
             "peak": imad_peak / 1e12, "unit": "TMAC/s", "frac": ach / (imad_peak / 1e12),
             "algorithmic_macs_per_launch": macs, "launch_ms": step_ms,
             "hbm_achieved_gbs": hbm, "hbm_algorithmic_bytes": 64 * self.n}
        return r, None

    def cpu(self, oracle, threads):
        sample = min(self.n, 1 << 20)
        vals = bytes(self.h_src.numpy().tobytes()[:sample * 32])
        t0 = time.perf_counter()
        oracle.ntt(vals, self.kind_name)
        ms = (time.perf_counter() - t0) * 1e3
        scale = (self.n * self.logn) / (sample * math.log2(sample))
        return None, ms * scale, (f"one 2^{int(math.log2(sample))} transform on 1 thread, scaled by n log n to "
                                  f"2^{self.logn}")


class SparseOp:
    def __init__(self, args):
        self.nb = 1 << args.log_n
        self.k = args.k
        self.metric = f"sparse G1 MSM k={args.k} over 2^{args.log_n} bases us"
        self.workload = (f"sparse-index G1 MSM: {args.k} indices without replacement from [0, 2^{args.log_n}) "
                         f"over resident [tau^i]G1 with precomputed window multiples (c = 8, setup), uniform Fr "
                         f"values")
        self.profile = "msm_g1_sparse"

    def setup(self, torch, b, s, rank):
        import numpy as np
        tau = torch.empty(32, dtype=torch.uint8, device="cuda")
        b.random_fr_device(2812, 1, tau.data_ptr(), s)
        powers = torch.empty(self.nb * 32, dtype=torch.uint8, device="cuda")
        b.fr_powers_device(tau.data_ptr(), self.nb, powers.data_ptr(), s)
        pts = torch.empty(self.nb * 64, dtype=torch.uint8, device="cuda")
        b.fixed_base_device(powers.data_ptr(), self.nb, False, pts.data_ptr(), s)
        torch.cuda.synchronize()
        self.h_bases = pts.cpu().numpy().tobytes()
        self.handle = b.register_bases(self.h_bases)
        # a resident SRS prepared for updates: 32 window multiples per base (c = 8)
        self.pre_c = b.precompute_bases(self.handle, 8)
        rng = np.random.default_rng(5150 + rank)
        self.idx = rng.choice(self.nb, size=self.k, replace=False).astype(np.uint64)
        self.d_idx = torch.from_numpy(self.idx.view(np.int64)).cuda()
        self.d_vals = torch.empty(self.k * 32, dtype=torch.uint8, device="cuda")
        b.random_fr_device(5151 + rank, self.k, self.d_vals.data_ptr(), s)
        torch.cuda.synchronize()
        self.tune_log = None
        self.config = {"bases": self.nb, "k": self.k, "precomputed_window_bits": self.pre_c}

    def step(self, b, s):
        return b.sparse_msm_device(self.handle, self.d_idx.data_ptr(), self.d_vals.data_ptr(), [0, self.k], stream=s)[0]

    def host_inputs(self, torch):
        self.h_vals = self.d_vals.cpu().numpy().tobytes()

    def e2e_step(self, dv, b):
        return b.sparse_msm_resident(self.handle, self.idx, self.h_vals, [0, self.k])[0]

    def e2e_bytes(self):
        return self.k * 40, 64

    def roofline(self, tl, imad_peak, step_ms):
        macs = msm_macs(self.k)
        ach = macs / (step_ms * 1e-3) / 1e12
        return ({"bound": "imad", "kernel": "whole sparse MSM (gather + Pippenger)", "achieved": ach,
                 "peak": imad_peak / 1e12, "unit": "TMAC/s", "frac": ach / (imad_peak / 1e12),
                 "algorithmic_macs_per_launch": macs, "launch_ms": step_ms}, None)

    def cpu(self, oracle, threads):
        vals = self.h_vals
        t0 = time.perf_counter()
        out = oracle.sparse_msm_g1(self.h_bases, self.idx, vals, threads=threads)
        return out, (time.perf_counter() - t0) * 1e3, f"one k={self.k} sparse MSM on the same inputs"


class FixedBaseOp:
    def __init__(self, args):
        self.n = 1 << args.log_n
        self.metric = f"fixed-base G1 2^{args.log_n} ms"
        self.workload = f"fixed-base [s_i]G1 for 2^{args.log_n} SRS exponents tau^i"
        self.profile = "fixed_base_g1"

    def setup(self, torch, b, s, rank):
        tau = torch.empty(32, dtype=torch.uint8, device="cuda")
        b.random_fr_device(2812 + rank, 1, tau.data_ptr(), s)
        self.sc = torch.empty(self.n * 32, dtype=torch.uint8, device="cuda")
        b.fr_powers_device(tau.data_ptr(), self.n, self.sc.data_ptr(), s)
        self.out = torch.empty(self.n * 64, dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        self.tune_log = None
        self.config = {"points": self.n}

    def step(self, b, s):
        b.fixed_base_device(self.sc.data_ptr(), self.n, False, self.out.data_ptr(), s)
        return None

    def host_inputs(self, torch):
        self.h_sc = torch.empty(self.n * 32, dtype=torch.uint8, pin_memory=True)
        self.h_sc.copy_(self.sc)
        self.h_out = torch.empty(self.n * 64, dtype=torch.uint8, pin_memory=True)

    def e2e_step(self, dv, b):
        err = ctypes.create_string_buffer(256)
        dst = ctypes.cast(ctypes.c_void_p(self.h_out.data_ptr()), ctypes.c_char_p)
        rc = dv.lib().dvgpu_bn254_fixed_base(b.handle, self.h_sc.data_ptr(), self.n, 0, dst, err, 256)
        if rc != 0:
            raise RuntimeError(err.value)
        return None

    def e2e_bytes(self):
        return self.n * 32, self.n * 64

    # the work convention of the 64 x 16 table (64 mixed adds a point), which
    # the 16-bit table beats by doing a quarter of the additions
    secondary_key = "convention_64_adds_roofline"

    def roofline(self, tl, imad_peak, step_ms):
        macs = self.n * (16 * G1_MADD_MACS + 10 * MAC_MUL)  # 16 mixed adds (16-bit signed windows) + warp-shared normalisation
        ach = macs / (step_ms * 1e-3) / 1e12
        conv = self.n * (64 * G1_MADD_MACS + 10 * MAC_MUL)
        conv_ach = conv / (step_ms * 1e-3) / 1e12
        return ({"bound": "imad", "kernel": "k_fb_generate", "achieved": ach, "peak": imad_peak / 1e12,
                 "unit": "TMAC/s", "frac": ach / (imad_peak / 1e12), "algorithmic_macs_per_launch": macs,
                 "launch_ms": step_ms},
                {"algorithmic_macs": conv, "achieved_tmacs": conv_ach, "frac": conv_ach / (imad_peak / 1e12),
                 "note": "64 mixed adds + normalisation per point, the 4-bit-window table's count"})

    def cpu(self, oracle, threads):
        sample = min(self.n, 1 << 16)
        t0 = time.perf_counter()
        oracle.fixed_base_g1(self.h_sc[:sample * 32], threads=threads)
        ms = (time.perf_counter() - t0) * 1e3
        return None, ms * self.n / sample, f"2^{int(math.log2(sample))} points, scaled linearly to the workload"


BN_R = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
BN_X = 4965661367192848881


def g2_check_fme(alg):
    """Fq multiplications per point of a subgroup check: G2 XYZZ doubling 27
    (9 Fq2 products), mixed addition 30, full addition 42, psi 6.
    Algorithm 1: [r]Q = 0; 2: psi(Q) = [6x^2]Q; 3: the seed-x Frobenius
    relation ([x]Q + Q + psi([x]Q) + psi^2([x]Q) = psi^3([2x]Q))."""
    if alg == 1:
        return 254 * 27 + bin(BN_R).count("1") * 30
    if alg == 2:
        lam = 6 * BN_X * BN_X
        return (lam.bit_length() - 1) * 27 + bin(lam).count("1") * 30 + 6 + 3 * 10
    return (BN_X.bit_length() - 1) * 27 + bin(BN_X).count("1") * 30 + 3 * 6 + 30 + 2 * 42 + 27 + 2 * 3 * 10


class G2CheckOp:
    """Batched G2 subgroup check over a corpus of 2^n wire points: half
    [s]G2 for uniform s (valid), half random twist points without cofactor
    clearing (invalid), all in one launch."""

    def __init__(self, args):
        self.n = 1 << args.log_n
        self.alg = args.alg
        self.metric = f"G2 subgroup check 2^{args.log_n} points ms (algorithm {args.alg})"
        self.workload = (f"2^{args.log_n} G2 wire points: half [s]G2 for uniform s, half random on-curve twist "
                         f"points without cofactor clearing; subgroup algorithm {args.alg}")
        self.profile = f"g2_check_2p{args.log_n}"

    def setup(self, torch, b, s, rank):
        half = self.n // 2
        sc = torch.empty(half * 32, dtype=torch.uint8, device="cuda")
        b.random_fr_device(4100 + rank, half, sc.data_ptr(), s)
        self.wire = torch.empty(self.n * 128, dtype=torch.uint8, device="cuda")
        b.fixed_base_device(sc.data_ptr(), half, True, self.wire.data_ptr(), s)
        b.random_twist_device(4200 + rank, self.n - half, self.wire.data_ptr() + 128 * half, s)
        self.masks = torch.empty(self.n, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        self.tune_log = None
        self.config = {"points": self.n, "valid": half, "algorithm": self.alg}

    def step(self, b, s):
        rep = b.g2_check_device(self.wire.data_ptr(), self.n, self.alg, self.masks.data_ptr(), s)
        return (rep.invalid_points, rep.first_invalid, rep.failure_mask)

    def host_inputs(self, torch):
        self.h_wire = torch.empty(self.n * 128, dtype=torch.uint8, pin_memory=True)
        self.h_wire.copy_(self.wire)
        self.h_masks = torch.empty(self.n, dtype=torch.int32, pin_memory=True)

    def e2e_step(self, dv, b):
        rep = dv.G2ValidationReport()
        err = ctypes.create_string_buffer(256)
        rc = dv.lib().dvgpu_bn254_g2_validation_inspect(b.handle, self.h_wire.data_ptr(), self.n, self.alg,
                                                         self.h_masks.data_ptr(), ctypes.byref(rep), err, 256)
        if rc not in (0, -5):  # -5: content rejected, report published (the reference's convention)
            raise RuntimeError(err.value)
        return (rep.invalid_points, rep.first_invalid, rep.failure_mask)

    def e2e_bytes(self):
        return self.n * 128, self.n * 4

    def roofline(self, tl, imad_peak, step_ms):
        macs = self.n * g2_check_fme(self.alg) * 136
        ach = macs / (step_ms * 1e-3) / 1e12
        return ({"bound": "imad", "kernel": "k_g2_check", "achieved": ach, "peak": imad_peak / 1e12,
                 "unit": "TMAC/s", "frac": ach / (imad_peak / 1e12), "algorithmic_macs_per_launch": macs,
                 "fme_per_point": g2_check_fme(self.alg), "launch_ms": step_ms}, None)

    def cpu(self, oracle, threads):
        import numpy as np
        sample = min(self.n, 1 << 13)
        wire = self.h_wire.numpy().tobytes()
        half = self.n // 2
        sub = wire[:64 * sample] + wire[128 * half:128 * half + 64 * sample]  # half valid, half invalid
        t0 = time.perf_counter()
        masks = oracle.g2_check(sub, self.alg, threads=threads)
        ms = (time.perf_counter() - t0) * 1e3
        gpu = self.h_masks.numpy()
        agree = bool(np.array_equal(masks[:sample // 2], gpu[:sample // 2]) and
                     np.array_equal(masks[sample // 2:], gpu[half:half + sample // 2]))
        self.cpu_agrees = agree
        return None, ms * self.n / sample, (f"{sample} points (half valid, half invalid) on {threads} threads, "
                                            f"scaled linearly; verdicts identical to the GPU's: {agree}")


def ecntt_macs(logn, rows):
    """Multiply-accumulates of a G1 transform: per stage, every butterfly
    costs two XYZZ additions and every butterfly with a twiddle other than 1
    a GLV scalar multiplication over signed 5-bit windows of its two 127-bit
    halves: the table of 1..16 multiples (8 doublings, 7 additions), then 26
    windows (125 doublings, two additions and one product beta X a window).
    A paired doubling is 7 products and 2 squares."""
    n = 1 << logn
    dbl = 7 * MAC_MUL + 2 * MAC_SQR
    smul = 8 * dbl + 7 * G1_ADD_MACS + 125 * dbl + 26 * (2 * G1_ADD_MACS + MAC_MUL)
    nontrivial = sum(rows * (n // 2 - (1 << s)) for s in range(logn))
    return rows * (n // 2) * logn * 2 * G1_ADD_MACS + nontrivial * smul


class EcNttOp:
    """G1 transform (EC-NTT) of rows of 2^12 points, the four-step packet
    length of the reference's rebuild (MAX_TRANSFORM_PACKET_LEN 4096)."""

    def __init__(self, args):
        self.logn = args.log_n
        self.rows = args.rows
        self.n = (1 << self.logn) * self.rows
        self.metric = f"G1 EC-NTT {self.rows} x 2^{self.logn} ms"
        self.workload = (f"G1 transform (arkworks radix-2 FFT over G1, rows normalised to affine) of {self.rows} "
                         f"rows of 2^{self.logn} points [s_i]G1, forward")
        self.profile = f"g1_ntt_{self.rows}x2p{self.logn}"

    def setup(self, torch, b, s, rank):
        sc = torch.empty(self.n * 32, dtype=torch.uint8, device="cuda")
        b.random_fr_device(8100 + rank, self.n, sc.data_ptr(), s)
        self.pts = torch.empty(self.n * 64, dtype=torch.uint8, device="cuda")
        b.fixed_base_device(sc.data_ptr(), self.n, False, self.pts.data_ptr(), s)
        self.out = torch.empty_like(self.pts)
        torch.cuda.synchronize()
        self.tune_log = None
        self.config = {"rows": self.rows, "row_len": 1 << self.logn, "points": self.n}

    def step(self, b, s):
        b.g1_ntt_rows_device(self.pts.data_ptr(), 1 << self.logn, self.rows, False, self.out.data_ptr(), s)
        return None

    def host_inputs(self, torch):
        self.h_pts = torch.empty(self.n * 64, dtype=torch.uint8, pin_memory=True)
        self.h_pts.copy_(self.pts)
        self.h_out = torch.empty(self.n * 64, dtype=torch.uint8, pin_memory=True)

    def e2e_step(self, dv, b):
        err = ctypes.create_string_buffer(256)
        dst = ctypes.cast(ctypes.c_void_p(self.h_out.data_ptr()), ctypes.c_char_p)
        rc = dv.lib().dvgpu_bn254_g1_ntt_rows(b.handle, self.h_pts.data_ptr(), 1 << self.logn, self.rows, 0, dst,
                                               err, 256)
        if rc != 0:
            raise RuntimeError(err.value)
        return None

    def e2e_bytes(self):
        return self.n * 64, self.n * 64

    def roofline(self, tl, imad_peak, step_ms):
        macs = ecntt_macs(self.logn, self.rows)
        ach = macs / (step_ms * 1e-3) / 1e12
        return ({"bound": "imad", "kernel": "k_ec_stage (all stages) + k_ec_store", "achieved": ach,
                 "peak": imad_peak / 1e12, "unit": "TMAC/s", "frac": ach / (imad_peak / 1e12),
                 "algorithmic_macs_per_launch": macs, "launch_ms": step_ms}, None)

    def cpu(self, oracle, threads):
        rows = min(self.rows, threads)
        pts = self.h_pts.numpy().tobytes()[:64 * rows << self.logn]
        t0 = time.perf_counter()
        out = oracle.g1_fft(pts, 1 << self.logn, False, threads=threads)
        ms = (time.perf_counter() - t0) * 1e3
        agree = out == self.h_out.numpy().tobytes()[:len(out)] if hasattr(self, "h_out") else None
        return None, ms * self.rows / rows, (f"{rows} rows on {rows} threads, scaled to {self.rows} rows; "
                                              f"identical to the GPU's: {agree}")


def serve_stream(sizes, count):
    """The seeded update stream: (session, distinct indices) per request."""
    import numpy as np
    rng = np.random.default_rng(5000)
    hot = [int(rng.integers(0, max(1, n - 64))) for n in sizes]
    out = []
    for t in range(count):
        j = int(rng.integers(len(sizes)))
        n = sizes[j]
        k = min(n, int(2 ** rng.uniform(0, 10)))
        if t % 2:
            k = min(k, 64)
            idx = hot[j] + rng.choice(64, size=k, replace=False)
        else:
            idx = rng.choice(n, size=k, replace=False)
        out.append((j, idx.astype(np.uint64)))
    return out


class ServeOp:
    """Serving: commitment updates from 64 resident sessions (n in
    {256, 4096, 65536} in ratio 37:18:9), supports of floor(2^U) entries,
    U ~ U[0, 10], capped at n, half in a 64-entry hotspot window per session,
    half uniform; fresh uniform values.  The same request stream runs through
    the served form (continuous batching, max_batch 64) and the per-call form
    (max_batch 1): all requests at once (saturation throughput) and as a
    Poisson stream at 80 % of the per-call capacity (latency)."""

    SIZES = [256] * 37 + [4096] * 18 + [65536] * 9

    def __init__(self, args):
        self.requests = args.requests
        self.metric = "served commitment updates/s (64 sessions, n 256/4096/65536)"
        self.workload = ("commitment updates C' = C + sum (v'_i - v_i) G_i over 64 resident sessions, "
                         f"{self.requests} requests, supports floor(2^U), U~U[0,10], half hotspot (64-entry window) "
                         "half uniform, uniform Fr values")
        self.profile = "serve"

    def _inputs(self, torch, b, s):
        self.sess = []
        for j, n in enumerate(self.SIZES):
            tau = torch.empty(32, dtype=torch.uint8, device="cuda")
            b.random_fr_device(7000 + j, 1, tau.data_ptr(), s)
            pw = torch.empty(n * 32, dtype=torch.uint8, device="cuda")
            b.fr_powers_device(tau.data_ptr(), n, pw.data_ptr(), s)
            pts = torch.empty(n * 64, dtype=torch.uint8, device="cuda")
            b.fixed_base_device(pw.data_ptr(), n, False, pts.data_ptr(), s)
            vals = torch.empty(n * 32, dtype=torch.uint8, device="cuda")
            b.random_fr_device(7100 + j, n, vals.data_ptr(), s)
            torch.cuda.synchronize()
            self.sess.append((pts.cpu().numpy().tobytes(), vals.cpu().numpy().tobytes()))
        reqs, total = [], 0
        for j, idx in serve_stream(self.SIZES, self.requests):
            reqs.append((j, idx, total, len(idx)))
            total += len(idx)
        vals = torch.empty(total * 32, dtype=torch.uint8, device="cuda")
        b.random_fr_device(7200, total, vals.data_ptr(), s)
        torch.cuda.synchronize()
        allv = vals.cpu().numpy().tobytes()
        self.reqs = [(j, idx, allv[32 * o:32 * (o + k)]) for j, idx, o, k in reqs]
        self.entries = total

    def _run(self, srv, max_batch, arrivals):
        """One pass of the request stream through a warm server: sessions
        (re)opened from the initial vectors, then the stream submitted at its
        arrival times (seconds from the start)."""
        srv.set_max_batch(max_batch)
        ids = [srv.open_session(p, v)[0] for p, v in self.sess]
        before = srv.stats()
        t0 = time.perf_counter()
        tickets = []
        for (j, idx, vals), at in zip(self.reqs, arrivals):
            while time.perf_counter() - t0 < at:
                pass
            tickets.append(srv.submit(ids[j], idx, vals))
        outs = [srv.wait(t) for t in tickets]
        wall = time.perf_counter() - t0
        st = srv.stats()
        for sid in ids:
            srv.close_session(sid)
        lat = sorted((r.done_ns - r.submit_ns) / 1e6 for _, r in outs)
        pct = lambda q: lat[min(len(lat) - 1, int(q * len(lat)))]
        # the slowest 1 %: time queued, time in their batch, batch sizes
        worst = sorted(outs, key=lambda o: o[1].done_ns - o[1].submit_ns)[-max(1, len(outs) // 100):]
        batch_ms = {}
        for _, r in outs:
            batch_ms[r.batch_id] = ((r.done_ns - r.start_ns) / 1e6, r.batch_requests)
        slowest_batch = max(batch_ms.values())
        tail = {"queued_ms": sum((r.start_ns - r.submit_ns) / 1e6 for _, r in worst) / len(worst),
                "in_batch_ms": sum((r.done_ns - r.start_ns) / 1e6 for _, r in worst) / len(worst),
                "batch_requests": [r.batch_requests for _, r in worst],
                "slowest_batch_ms": slowest_batch[0], "slowest_batch_requests": slowest_batch[1]}
        return {"commitments": [c for c, _ in outs], "wall_s": wall, "per_s": len(outs) / wall,
                "p50_ms": pct(0.50), "p99_ms": pct(0.99), "max_ms": lat[-1], "mean_ms": sum(lat) / len(lat),
                "batches": st.batches - before.batches, "largest_batch": max(r.batch_requests for _, r in outs)}

    def run_standalone(self, args, torch, dv, b, s, sampler, imad_peak_fn, world=1):
        import numpy as np
        self._inputs(torch, b, s)
        zeros = [0.0] * self.requests
        srv = dv.DvgpuServer(150 << 30, 64)
        self._run(srv, 64, zeros)  # warm-up: workspaces reach their working size
        self._run(srv, 1, zeros[:200])
        sampler.start()
        launches0 = b.launch_count()
        sat_served = self._run(srv, 64, zeros)
        launches = b.launch_count() - launches0
        sat_plain = self._run(srv, 1, zeros)
        rate = 0.8 * sat_plain["per_s"]
        arrivals = np.cumsum(np.random.default_rng(5001).exponential(1.0 / rate, self.requests)).tolist()
        poi_served = self._run(srv, 64, arrivals)
        poi_plain = self._run(srv, 1, arrivals)
        clocks = sampler.stop()
        srv.close()
        runs = (sat_served, sat_plain, poi_served, poi_plain)
        exact = all(r["commitments"] == sat_served["commitments"] for r in runs)
        # final commitment of every session = full recommitment of its final vector
        vecs = [bytearray(v) for _, v in self.sess]
        last = {}
        for t, (j, idx, vals) in enumerate(self.reqs):
            for q, i in enumerate(idx):
                vecs[j][32 * int(i):32 * (int(i) + 1)] = vals[32 * q:32 * (q + 1)]
            last[j] = sat_served["commitments"][t]
        for j, c in last.items():
            exact = exact and b.msm(self.sess[j][0], bytes(vecs[j])) == c
        macs = sum(msm_macs(len(idx)) for _, idx, _ in self.reqs)
        ach = macs / sat_served["wall_s"] / 1e12
        peak = imad_peak_fn() / 1e12
        strip = lambda r: {k: v for k, v in r.items() if k != "commitments"}
        # N replicas (one server per GPU): whole-job rate over the slowest rank's saturation run
        job_per_s = world * self.requests / max_over_ranks(sat_served["wall_s"], world)
        line = {
            "metric": self.metric, "value": job_per_s, "unit": "updates/s", "n_gpus": world,
            "steps": self.requests, "warmup": 1, "ms_per_step": 1e3 / sat_served["per_s"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32 limbs (Fq/Fr Montgomery, exact)",
            "data": "synthetic",
            "config": {"workload": self.workload, "op": "serve",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "sessions": len(self.SIZES), "requests": self.requests, "entries": self.entries,
                       "l2": "not flushed: a stream of small requests against resident sessions"},
            "e2e": {"value": job_per_s, "unit": "updates/s",
                    "h2d_bytes_per_step": 40 * self.entries / self.requests, "d2h_bytes_per_step": 64,
                    "call": "dvgpu_serve_submit/wait from host memory (the serving API is host-to-host)"},
            "serving": {"saturation": {"served": strip(sat_served), "per_call": strip(sat_plain),
                                       "speedup": sat_served["per_s"] / sat_plain["per_s"]},
                        "poisson": {"rate_per_s": rate, "served": strip(poi_served), "per_call": strip(poi_plain)},
                        "bit_exact": exact,
                        "note": "commitment updates only: the update proofs of the reference protocol are not "
                                "built"},
            "roofline": {"bound": "imad", "kernel": "all launches of the saturation run (sparse delta MSMs)",
                         "achieved": ach, "peak": peak, "unit": "TMAC/s", "frac": ach / peak,
                         "algorithmic_macs_per_launch": macs, "traffic": None},
            "gpu_launches": launches, "clocks": clocks,
        }
        if not args.no_cpu_baseline and world == 1:
            from oracle import oracle
            threads = os.cpu_count() or 1
            sample = self.reqs[:200]
            t0 = time.perf_counter()
            for j, idx, vals in sample:
                oracle.sparse_msm_g1(self.sess[j][0], idx, vals, threads=threads)
            cpu_s = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": len(sample) / cpu_s, "unit": "updates/s", "cores": threads,
                                    "kind": "port", "sample": f"the first {len(sample)} requests' sparse MSMs"}
        return line


R_FR = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001


def valid_witness(n, seed):
    """A uniform valid ToyCircuit(n) instance (toy_circuit.rs:45-90): left,
    right and multiplier uniform in Fr per gate; sum and product follow."""
    import random
    rng = random.Random(seed)
    pub, w = [0] * n, [0] * (6 * n)
    for i in range(n):
        left, right, mul = rng.randrange(R_FR), rng.randrange(R_FR), rng.randrange(R_FR)
        s = (left + right) % R_FR
        pub[i] = left
        w[i], w[n + i], w[2 * n + i], w[3 * n + i], w[4 * n + i], w[5 * n + i] = left, right, s, s, mul, s * mul % R_FR
    return pub, w


def bench_trapdoors(sizes, seed=9900):
    """Seeded trapdoor pairs per circuit size, drawn until they meet the
    setup's rejection rules (srs.rs:158-178): nonzero, distinct, outside the
    8n-point domain, tau_x != tau_y^8."""
    import random
    rng = random.Random(seed)
    out = {}
    for n in sorted(set(sizes)):
        m = 8 * n
        while True:
            tx, ty = rng.randrange(1, R_FR), rng.randrange(1, R_FR)
            if tx != ty and pow(tx, m, R_FR) != 1 and pow(ty, m, R_FR) != 1 and tx != pow(ty, 8, R_FR):
                out[n] = (tx, ty)
                break
    return out


class ProofsCpu:
    """The CPU restatement of the reference's sparse update path (oracle,
    bases route: sparse MSMs over the SRS points, the subproduct tree, FFT
    products and exact division, then the pairing verifier) on the GPU
    arm's own request stream, in order.  Setup is not timed: per distinct n
    the SRS points and one session on the sessions' common initial witness,
    whose anchor and opening cache come from the trapdoor scalars (identical
    values).  Each request goes to the CPU session of its n (updates rewrite
    s5 and s6 = s4 u only, so every one stays valid there).  Updates that
    re-anchor are left out of the rate (on the CPU the dense anchor and its
    opening cache take minutes at n = 65536), so the rate counts sparse
    proofs only."""

    def __init__(self, op, threads):
        from oracle import dynaverse as D
        self.sessions = {}
        traps = bench_trapdoors(op.sizes)
        for n in sorted(set(op.sizes)):
            tx, ty = traps[n]
            P = D.Params(n, tx, ty, "bases", threads=threads)
            pub, w = op.wit[op.sizes.index(n)]
            self.sessions[n] = D.Session(P, pub, w, verify=False, scalar_anchors=True)
        self.sizes = op.sizes
        self.reqs = op.reqs
        self.pos = 0
        self.rebuilds = 0
        self.count = 0

    def sample(self, budget_s):
        """Sparse proofs/s over the next requests, until budget_s of timed work."""
        times = []
        while self.pos < len(self.reqs) and sum(times) < budget_s:
            j, idx, vals = self.reqs[self.pos]
            self.pos += 1
            S = self.sessions[self.sizes[j]]
            values = [int.from_bytes(vals[32 * i:32 * i + 32], "little") for i in range(len(idx))]
            t0 = time.perf_counter()
            S.update(idx, values, verify=True)
            dt = time.perf_counter() - t0
            if S.last_rebuilt:
                self.rebuilds += 1
            else:
                times.append(dt)
        self.count += len(times)
        return (len(times) / sum(times)) if times else None

    def describe(self):
        ns = "/".join(str(n) for n in sorted(self.sessions))
        return (f"{self.count} sparse update proofs (n = {ns}): the benchmark's own request stream in order, each "
                f"proved by the oracle's restatement of the reference's steps and verified with its pairing checks "
                f"({self.rebuilds} re-anchoring updates left out)")


def proof_probe(dv, kind, n):
    """A fixed case of the update-proof pipeline for profiler captures.
    k_accum launches: two per session open (G1, G2 sets), then per batch m1,
    m3 (G2), m2 and md (the dense sets) -- so 'update' has md at k_accum
    launch 7 and 'batch' at 131."""
    import threading
    import numpy as np
    sessions, batch = (2, 1) if kind == "update" else (64, 64)
    e = dv.DynaverseEngine(100 << 30, batch)
    tx, ty = bench_trapdoors([n])[n]
    ph = e.params_create(n, tx, ty)
    enc = lambda xs: b"".join(v.to_bytes(32, "little") for v in xs)
    pub, w = valid_witness(n, 9000)
    pb, wb = enc(pub), enc(w)
    ids = [e.open_session(ph, pb, wb)[0] for _ in range(sessions)]
    rng = np.random.default_rng(5)
    reqs = []
    for sid in ids[:batch]:
        g = 64 if kind == "update" else int(2 ** rng.uniform(0, 6))
        idx, vals = [], []
        for gate in rng.choice(n, size=g, replace=False).tolist():
            u = int(rng.integers(1, 1 << 62))
            idx += [4 * n + gate, 5 * n + gate]
            vals += [u, w[3 * n + gate] * u % R_FR]
        reqs.append((sid, idx, enc(vals)))
    busy = None
    if kind == "batch":
        # a parameter build holds the engine's worker while all 64 requests queue
        n2 = n // 4
        tx2, ty2 = bench_trapdoors([n2])[n2]
        busy = threading.Thread(target=lambda: e.params_create(n2, tx2, ty2))
        busy.start()
        time.sleep(0.01)
    outs = [e.wait(t) for t in [e.submit(sid, idx, v) for sid, idx, v in reqs]]
    if busy:
        busy.join()
    st = e.stats()
    print(json.dumps({"probe": kind, "n": n, "batches": len(set(r.batch_id for _, r in outs)),
                      "batch_ms": (outs[0][1].done_ns - outs[0][1].start_ns) / 1e6,
                      "dense_accum_ms": st.dense_accum_ns / 1e6, "dense_accum_adds": st.dense_accum_adds}))
    e.close()


def operator_points(torch, dv, b, s, imad_peak, threads, with_cpu=True):
    """The operator targets beside the proof rate: a plain 2^20-point G1 MSM
    (bases and scalars passed on every call, dvgpu_bn254_msm, as the
    reference's OperatorBackend::msm does) and a 2^22 forward Fr NTT.  Each:
    device time with inputs resident and L2 flushed between steps (CUDA
    events on the launching stream, mean of 20 after 3 warm-ups), end to end
    through the C-ABI from pinned host buffers, the fraction of the measured
    IMAD peak, and the CPU oracle on the same inputs with the results
    compared."""
    import types
    from oracle import oracle
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def timed(fn, steps=20, warm=3):
        for _ in range(warm):
            r = fn()
        torch.cuda.synchronize()
        total = 0.0
        for _ in range(steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = fn()
            e1.record(stream)
            e1.synchronize()
            total += e0.elapsed_time(e1)
        return total / steps, r

    def wall(fn, steps):
        fn()
        t0 = time.perf_counter()
        for _ in range(steps):
            fn()
        return (time.perf_counter() - t0) * 1e3 / steps

    out = {}
    m = MsmOp(types.SimpleNamespace(log_n=20, kind="forward"))
    m.setup(torch, b, s, 0)
    ms, res = timed(lambda: m.step(b, s))
    m.host_inputs(torch)
    e2e = wall(lambda: m.e2e_step(dv, b), 10)
    macs = msm_macs(m.n)
    d = {"call": "dvgpu_bn254_msm (plain: bases and scalars from host memory every call)", "points": m.n,
         "window_bits": m.tuned_c, "device_ms": ms, "e2e_ms": e2e,
         "h2d_bytes": m.n * 96, "d2h_bytes": 64 + m.config["windows"] * 128,
         "roofline": {"bound": "imad", "achieved": macs / (ms * 1e-3) / 1e12, "peak": imad_peak / 1e12,
                      "unit": "TMAC/s", "frac": macs / (ms * 1e-3) / imad_peak,
                      "convention": "min_c ceil(254/c)(n mixed + 2^c full XYZZ additions); a mixed addition 8 x 136 + 2 x 108 MACs, a full one 12 x 136 + 2 x 108"}}
    if with_cpu:
        cpu_out, cpu_ms, _ = m.cpu(oracle, threads)
        d["cpu_oracle"] = {"ms": cpu_ms, "cores": threads, "matches_gpu": cpu_out == res}
    out["msm_g1_2p20"] = d
    del m
    t = NttOp(types.SimpleNamespace(log_n=22, kind="forward"))
    t.setup(torch, b, s, 0)
    ms, _ = timed(lambda: t.step(b, s))
    t.host_inputs(torch)
    e2e = wall(lambda: t.e2e_step(dv, b), 5)
    macs = t.fme() * 136
    d = {"call": "dvgpu_bn254_ntt_ex (forward)", "elements": t.n, "device_ms": ms, "e2e_ms": e2e,
         "h2d_bytes": 32 * t.n, "d2h_bytes": 32 * t.n,
         "roofline": {"bound": "imad", "achieved": macs / (ms * 1e-3) / 1e12, "peak": imad_peak / 1e12,
                      "unit": "TMAC/s", "frac": macs / (ms * 1e-3) / imad_peak,
                      "convention": "(n/2) log2 n Fr products x 136 MACs",
                      "hbm_gbs": 64 * t.n / (ms * 1e-3) / 1e9}}
    if with_cpu:
        vals = bytes(t.h_src.numpy().tobytes())
        t0 = time.perf_counter()
        ref = oracle.ntt(vals, "forward")
        d["cpu_oracle"] = {"ms": (time.perf_counter() - t0) * 1e3, "cores": 1,
                           "matches_gpu": ref == bytes(t.dst.cpu().numpy().tobytes())}
    out["ntt_2p22"] = d
    return out


def proof_stream(sizes, witnesses, count, umax, seed):
    """The seeded update stream of the serving workload: a session, a support
    of floor(2^U) gates (U ~ U[0, umax], capped at n), half in the session's
    64-gate hotspot window and half uniform over [0, n), every gate given a
    fresh uniform s5 value u and s6 = s4 u so the circuit stays valid."""
    import random
    import numpy as np
    rng = np.random.default_rng(seed)
    vr = random.Random(seed + 1)
    hot = [int(rng.integers(0, max(1, n - 64))) for n in sizes]
    out = []
    for t in range(count):
        j = int(rng.integers(len(sizes)))
        n = sizes[j]
        g = min(n, int(2 ** rng.uniform(0, umax)))
        if t % 2:
            gates = hot[j] + rng.choice(min(64, n), size=min(g, 64, n), replace=False)
        else:
            gates = rng.choice(n, size=g, replace=False)
        w = witnesses[j]
        idx, vals = [], []
        for gate in gates.tolist():
            u = vr.randrange(R_FR)
            idx += [4 * n + gate, 5 * n + gate]
            vals += [u, w[3 * n + gate] * u % R_FR]
        out.append((j, idx, b"".join(v.to_bytes(32, "little") for v in vals)))
    return out


class ProofServeOp:
    """Dynaverse update proofs (row a10): sessions of ToyCircuit(n) with
    resident parameters and state; a stream of sparse witness updates; each
    request returns a complete DynaverseProof, verified on the device before
    it is published (the reference session verifies each proof too,
    session.rs:126-131).  The same stream runs through the served form
    (continuous batching, max_batch 64) and the per-call form (max_batch 1:
    one update at a time, each a full pipeline with its own launches), at
    saturation (all requests queued at once) and as a Poisson stream at 80 %
    of the per-call capacity (latency).  Proofs are identical between the
    forms.  Default: 64 sessions of n = 65536; --mix: 64 sessions with
    n in {256, 4096, 65536} in ratio 37:18:9."""

    def __init__(self, args):
        self.mix = args.mix
        n = 1 << args.log_n
        self.sizes = [256] * 37 + [4096] * 18 + [65536] * 9 if args.mix else [n] * args.sessions
        self.requests = args.requests
        self.umax = args.umax
        label = "n 256/4096/65536 mix" if args.mix else f"n={n}"
        self.metric = f"update proofs/s ({label}, served, every proof verified)"
        self.workload = (f"Dynaverse update proofs over {len(self.sizes)} sessions ({label}), {self.requests} requests; "
                         f"supports of 2 floor(2^U) witness indices (floor(2^U) multiplication gates, wires s5 and s6), "
                         f"U~U[0,{self.umax}], half in a 64-gate hotspot window, half "
                         "uniform; every gate's s5 a fresh uniform Fr and s6 = s4 s5; re-anchor when the delta "
                         "reaches ceil(sqrt(n)) (session.rs:92)")
        self.profile = "dynaverse_serve"

    def config(self, world):
        return {"workload": self.workload, "op": "proofs",
                "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                "sessions": len(self.sizes), "requests": self.requests,
                "l2": "not flushed: a stream of requests against resident sessions"}

    def _setup(self, dv):
        import random
        self.eng = dv.DynaverseEngine(150 << 30, 64)
        self.params = {n: self.eng.params_create(n, tx, ty) for n, (tx, ty) in bench_trapdoors(self.sizes).items()}
        self._inputs()

    def _inputs(self):
        # sessions of one size open on the same seeded witness (their states
        # then diverge), so the stream is valid on the CPU arm's one session
        # per size and both arms process the same requests
        by_n = {n: valid_witness(n, 9000 + n.bit_length()) for n in sorted(set(self.sizes))}
        enc = {n: (b"".join(v.to_bytes(32, "little") for v in p), b"".join(v.to_bytes(32, "little") for v in w))
               for n, (p, w) in by_n.items()}
        self.wit = [by_n[n] for n in self.sizes]
        self.pub_b = [enc[n][0] for n in self.sizes]
        self.wit_b = [enc[n][1] for n in self.sizes]
        self.reqs = proof_stream(self.sizes, [w for _, w in self.wit], self.requests, self.umax, 9100)

    def _run(self, max_batch, arrivals):
        e = self.eng
        e.set_max_batch(max_batch)
        ids = [e.open_session(self.params[n], self.pub_b[j], self.wit_b[j])[0] for j, n in enumerate(self.sizes)]
        before = e.stats()
        t0 = time.perf_counter()
        tickets = []
        for (j, idx, vals), at in zip(self.reqs, arrivals):
            while time.perf_counter() - t0 < at:
                pass
            tickets.append(e.submit(ids[j], idx, vals))
        outs = [e.wait(t) for t in tickets]
        wall = time.perf_counter() - t0
        st = e.stats()
        for sid in ids:
            e.close_session(sid)
        lat = sorted((r.done_ns - r.submit_ns) / 1e6 for _, r in outs)
        pct = lambda q: lat[min(len(lat) - 1, int(q * len(lat)))]
        # the slowest 1 %: time queued, time in their batch, batch sizes
        worst = sorted(outs, key=lambda o: o[1].done_ns - o[1].submit_ns)[-max(1, len(outs) // 100):]
        batch_ms = {}
        for _, r in outs:
            batch_ms[r.batch_id] = ((r.done_ns - r.start_ns) / 1e6, r.batch_requests)
        slowest_batch = max(batch_ms.values())
        tail = {"queued_ms": sum((r.start_ns - r.submit_ns) / 1e6 for _, r in worst) / len(worst),
                "in_batch_ms": sum((r.done_ns - r.start_ns) / 1e6 for _, r in worst) / len(worst),
                "batch_requests": [r.batch_requests for _, r in worst],
                "slowest_batch_ms": slowest_batch[0], "slowest_batch_requests": slowest_batch[1]}
        return {"proofs": [p for p, _ in outs], "wall_s": wall, "per_s": len(outs) / wall,
                "p50_ms": pct(0.50), "p99_ms": pct(0.99), "max_ms": lat[-1], "mean_ms": sum(lat) / len(lat),
                "batches": st.batches - before.batches, "largest_batch": max(r.batch_requests for _, r in outs),
                "rebuilds": sum(r.rebuilt for _, r in outs), "launches": st.launches - before.launches,
                "msm_fme": st.msm_fme - before.msm_fme, "host_ms": (st.host_ns - before.host_ns) / 1e6,
                "device_wait_ms": (st.device_wait_ns - before.device_wait_ns) / 1e6,
                "dense_accum_ms": (st.dense_accum_ns - before.dense_accum_ns) / 1e6,
                "dense_accum_adds": st.dense_accum_adds - before.dense_accum_adds,
                "allocations": st.allocations - before.allocations,
                "allocation_ms": (st.allocation_ns - before.allocation_ns) / 1e6,
                "enqueue_ms": (st.enqueue_ns - before.enqueue_ns) / 1e6,
                "slowest_alloc": {"ms": st.slowest_alloc_ns / 1e6, "bytes": st.slowest_alloc_bytes,
                                  "pinned": bool(st.slowest_alloc_pinned)}, "tail": tail}

    def run_standalone(self, args, torch, dv, b, s, sampler, imad_peak_fn, world=1):
        import numpy as np
        self._setup(dv)
        zeros = [0.0] * self.requests
        # warm-up: the whole stream once served (workspaces, tables, NTT plans
        # and the re-anchor buffer pool reach their sizes), a few per call
        self._run(64, zeros)
        self._run(1, zeros[:8])
        sampler.start()
        sat_served = self._run(64, zeros)
        sat_plain = self._run(1, zeros)
        rate = 0.8 * sat_plain["per_s"]
        arrivals = np.cumsum(np.random.default_rng(9200).exponential(1.0 / rate, self.requests)).tolist()
        poi_served = self._run(64, arrivals)
        poi_plain = self._run(1, arrivals)
        clocks = sampler.stop()
        runs = (sat_served, sat_plain, poi_served, poi_plain)
        exact = all(r["proofs"] == sat_served["proofs"] for r in runs)
        # every proof was verified before publication; re-check a sample with the device verifier
        e = self.eng
        sample_ok = True
        for (j, _, _), proof in list(zip(self.reqs, sat_served["proofs"]))[:32]:
            sample_ok &= e.verify(self.params[self.sizes[j]], self.pub_b[j], proof)
        peak = imad_peak_fn() / 1e12
        macs = sat_served["msm_fme"] * 136
        ach = macs / sat_served["wall_s"] / 1e12
        # the dominant kernel: the dense MSMs' bucket accumulation, timed live
        acc_macs = sat_served["dense_accum_adds"] * G1_MADD_MACS
        acc_ach = acc_macs / max(1e-9, sat_served["dense_accum_ms"] * 1e-3) / 1e12
        strip = lambda r: {k: v for k, v in r.items() if k != "proofs"}
        job_per_s = world * self.requests / max_over_ranks(sat_served["wall_s"], world)
        in_bytes = sum(8 * len(idx) + len(vals) for _, idx, vals in self.reqs) / self.requests
        line = {
            "metric": self.metric, "value": job_per_s, "unit": "proofs/s", "n_gpus": world,
            "steps": self.requests, "warmup": 1, "ms_per_step": 1e3 / sat_served["per_s"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32 limbs (Fq/Fr Montgomery, exact)",
            "data": "synthetic (seeded trapdoors, uniform valid witnesses, seeded update stream)",
            "config": self.config(world),
            "e2e": {"value": job_per_s, "unit": "proofs/s", "h2d_bytes_per_step": in_bytes,
                    "d2h_bytes_per_step": 9304,
                    "call": "dvgpu_dynaverse_submit/wait from host memory (update in, proof out)"},
            "serving": {"saturation": {"served": strip(sat_served), "per_call": strip(sat_plain),
                                       "speedup": sat_served["per_s"] / sat_plain["per_s"]},
                        "poisson": {"rate_per_s": rate, "served": strip(poi_served), "per_call": strip(poi_plain),
                                    "p99_ratio": poi_plain["p99_ms"] / poi_served["p99_ms"]},
                        "bit_exact": exact, "device_verifier_sample_accepted": bool(sample_ok)},
            "roofline": {"bound": "imad",
                         "kernel": "k_accum of the dense MSMs (anchor openings, re-anchor quotients; c = 16 table)",
                         "achieved": acc_ach, "peak": peak, "unit": "TMAC/s", "frac": acc_ach / peak,
                         "peak_source": "dvgpu_probe_imad_rate, measured in this run",
                         "algorithmic_macs_per_launch": acc_macs / max(1, sat_served["batches"]),
                         "launch_ms": sat_served["dense_accum_ms"] / max(1, sat_served["batches"]),
                         "convention": "8 Fq products x 136 + 2 Fq squares x 108 MACs per XYZZ mixed addition, 16 per dense term",
                         "traffic": (None if load_traffic("dynaverse_dense_accum", "traffic_bytes_per_add") is None
                                     else load_traffic("dynaverse_dense_accum", "traffic_bytes_per_add") *
                                     sat_served["dense_accum_adds"] / max(1, sat_served["batches"])),
                         "traffic_note": ("DRAM bytes per mixed addition of a captured 64-job launch "
                                          "(profiles/dynaverse_dense_accum.txt) x this run's additions per launch")},
            "msm_whole_run": {"achieved": ach, "frac": ach / peak, "algorithmic_macs": macs,
                              "convention": "sum over MSM sets of min_c ceil(254/c)(10k + 14 2^c) Fq products x 136 (x3 G2; squares counted as products), "
                                            "over the saturation run's wall time"},
            "gpu_launches": sat_served["launches"], "clocks": clocks,
        }
        self.eng.close()
        if world == 1 and not args.no_operators:
            line["operators"] = operator_points(torch, dv, b, s, peak * 1e12, os.cpu_count() or 1,
                                                with_cpu=not args.no_cpu_baseline)
        if not args.no_cpu_baseline and world == 1:
            threads = os.cpu_count() or 1
            cpu = ProofsCpu(self, threads)
            rate = cpu.sample(20.0)
            if rate is not None:
                line["cpu_baseline"] = {"value": rate, "unit": "proofs/s", "cores": threads, "kind": "port",
                                        "sample": cpu.describe()}
        return line


def batch_workload(log_bases):
    """The batching workload: 512 G1 MSMs of floor(2^U) points, U ~ U[8, 18],
    over prefixes of the SRS, and 256 forward NTTs of 2^floor(U) elements,
    U ~ U[10, 20] (seeded)."""
    import numpy as np
    rng = np.random.default_rng(4004)
    sizes = [min(1 << log_bases, int(2 ** u)) for u in rng.uniform(8, 18, 512)]
    logs = [int(u) for u in rng.uniform(10, 20, 256)]
    return sizes, logs


def batch_macs(sizes, logs):
    return sum(msm_macs(n) for n in sizes) + sum((1 << L) // 2 * L for L in logs) * MAC_MUL


def batch_cpu(oracle, threads, bases, sizes, logs, scalars, ntt_vals):
    """CPU oracle on a bounded sample of the batch (MSMs in order until 2^20
    points, on all threads; the first 8 NTTs on 1 thread), scaled to the
    whole batch by algorithmic multiply-accumulates."""
    msm_t, msm_done, off, k = 0.0, 0, 0, 0
    while k < len(sizes) and (k == 0 or sum(sizes[:k]) < (1 << 20)):
        n = sizes[k]
        t0 = time.perf_counter()
        oracle.msm_g1(bases[:64 * n], scalars[32 * off:32 * (off + n)], threads=threads)
        msm_t += time.perf_counter() - t0
        msm_done += msm_macs(n)
        off += n
        k += 1
    ntt_t, ntt_macs, noff = 0.0, 0, 0
    for L in logs[:8]:
        n = 1 << L
        t0 = time.perf_counter()
        oracle.ntt(ntt_vals[32 * noff:32 * (noff + n)], "forward")
        ntt_t += time.perf_counter() - t0
        ntt_macs += n // 2 * L * 136
        noff += n
    all_msm = sum(msm_macs(n) for n in sizes)
    all_ntt = sum((1 << L) // 2 * L for L in logs) * 136
    ms = (msm_t * all_msm / msm_done + ntt_t * all_ntt / ntt_macs) * 1e3
    return ms, (f"{k} MSMs ({sum(sizes[:k])} points, {threads} threads) and 8 NTTs (1 thread), scaled to the "
                f"whole batch by algorithmic multiply-accumulates")


class BatchOp:
    """Batching: 512 uneven G1 MSMs over a resident SRS plus 256 uneven NTTs
    per step, as one replay of a CUDA-graph batch plan (per-class launch
    sequences over precomputed tables, NTTs in one persistent launch),
    compared with the plain per-call loop on the same GPU and inputs."""

    LOG_BASES = 18

    def __init__(self, args):
        self.sizes, self.logs = batch_workload(self.LOG_BASES)
        self.metric = "batch of 512 G1 MSMs (2^8..2^18) + 256 NTTs (2^10..2^20) ms"
        self.workload = ("512 G1 MSMs of floor(2^U) points, U~U[8,18], over prefixes of a resident 2^18 SRS "
                         "[tau^i]G1, uniform Fr scalars; 256 forward Fr NTTs of 2^floor(U), U~U[10,20]; one "
                         "replay of a CUDA-graph batch plan (plan creation, autotuning and tables are setup)")
        self.profile = "batch_plan"

    def setup(self, torch, b, s, rank):
        nb = 1 << self.LOG_BASES
        tau = torch.empty(32, dtype=torch.uint8, device="cuda")
        b.random_fr_device(2812, 1, tau.data_ptr(), s)
        powers = torch.empty(nb * 32, dtype=torch.uint8, device="cuda")
        b.fr_powers_device(tau.data_ptr(), nb, powers.data_ptr(), s)
        pts = torch.empty(nb * 64, dtype=torch.uint8, device="cuda")
        b.fixed_base_device(powers.data_ptr(), nb, False, pts.data_ptr(), s)
        torch.cuda.synchronize()
        self.h_points = torch.empty(nb * 64, dtype=torch.uint8, pin_memory=True)
        self.h_points.copy_(pts)
        self.handle = b.register_bases(self.h_points.numpy().tobytes())
        self.plan, self.tune_log = b.batch_plan_create(self.handle, self.sizes, self.logs)
        self.buf = b.batch_plan_buffers(self.plan)
        self.total = sum(self.sizes)
        self.ntt_elems = sum(1 << L for L in self.logs)
        b.random_fr_device(2813 + rank, self.total, self.buf.scalars, s)
        b.random_fr_device(3000 + rank, self.ntt_elems, self.buf.ntt_values, s)
        torch.cuda.synchronize()
        self.config = {"msms": len(self.sizes), "msm_points_total": self.total,
                       "msm_sizes": [min(self.sizes), max(self.sizes)], "ntts": len(self.logs),
                       "ntt_elements_total": self.ntt_elems, "ntt_logs": [min(self.logs), max(self.logs)],
                       "msm_classes": [{"sets": c["sets"], "c": c["best_c"], "seg": c.get("best_seg")}
                                       for c in self.tune_log["classes"]],
                       "ntt_radix": self.tune_log["ntt"].get("best_radix"),
                       "ntt_tile": self.tune_log["ntt"].get("best_tile"),
                       "graph_nodes": self.buf.graph_nodes, "graph_kernels": self.buf.graph_kernels}
        self.launches_per_step = self.buf.graph_kernels
        # library kernels run so far (captured launches did not run): a
        # profiler skips these plus the warm-up replays to reach a replay
        self.config["setup_launches"] = b.launch_count() - self.buf.graph_kernels

    def step(self, b, s):
        b.batch_plan_launch(self.plan, s)
        return None

    def host_inputs(self, torch):
        import ctypes as C
        self._b.batch_plan_check(self.plan)  # the timed replays had valid inputs
        self.h_scalars = torch.empty(self.total * 32, dtype=torch.uint8, pin_memory=True)
        self.h_ntt = torch.empty(self.ntt_elems * 32, dtype=torch.uint8, pin_memory=True)
        self.h_scalars.copy_(device_view(torch, self.buf.scalars, self.buf.scalar_bytes))
        self.h_ntt.copy_(device_view(torch, self.buf.ntt_values, self.buf.ntt_bytes))
        self.h_msm_out = torch.empty(64 * len(self.sizes), dtype=torch.uint8, pin_memory=True)
        self.h_ntt_out = torch.empty(self.ntt_elems * 32, dtype=torch.uint8, pin_memory=True)
        self.graph_msm = device_view(torch, self.buf.msm_results, self.buf.msm_result_bytes).cpu().numpy().tobytes()
        self.graph_ntt = device_view(torch, self.buf.ntt_results, self.buf.ntt_bytes).clone()

    def extra(self, torch, dv, b, s):
        """The plain per-call loop on the same GPU and inputs: device-resident
        (dvgpu_bn254_msm_resident without precomputed tables + ntt_device per
        transform) and reference-facing with host buffers (dvgpu_bn254_msm,
        dvgpu_bn254_ntt_ex per call).  Both must reproduce the graph's
        results bit for bit."""
        err = ctypes.create_string_buffer(256)
        d_sc = self.buf.scalars
        d_in = self.buf.ntt_values
        ref_ntt = torch.empty(self.ntt_elems * 32, dtype=torch.uint8, device="cuda")

        def device_loop():
            outs, off = [], 0
            for n in self.sizes:
                outs.append(b.msm_resident(self.handle, d_sc + 32 * off, n, stream=s))
                off += n
            off = 0
            for L in self.logs:
                b.ntt_device(d_in + 32 * off, 1 << L, 0, ref_ntt.data_ptr() + 32 * off, s)
                off += 1 << L
            torch.cuda.synchronize()
            return outs

        outs = device_loop()  # warm-up (window tables, NTT tables)
        t0 = time.perf_counter()
        outs = device_loop()
        per_call_ms = (time.perf_counter() - t0) * 1e3
        exact = b"".join(outs) == self.graph_msm and bool(torch.equal(ref_ntt, self.graph_ntt))
        L = dv.lib()
        cast = lambda p: ctypes.cast(ctypes.c_void_p(p), ctypes.c_char_p)
        out = ctypes.create_string_buffer(64)
        h_out = torch.empty(self.ntt_elems * 32, dtype=torch.uint8, pin_memory=True)

        def host_loop():
            res, off = [], 0
            for n in self.sizes:
                if L.dvgpu_bn254_msm(b.handle, self.h_points.data_ptr(), self.h_scalars.data_ptr() + 32 * off, n,
                                     out, err, 256) != 0:
                    raise RuntimeError(err.value)
                res.append(out.raw)
                off += n
            off = 0
            for Lg in self.logs:
                if L.dvgpu_bn254_ntt_ex(b.handle, self.h_ntt.data_ptr() + 32 * off, 1 << Lg, 0,
                                        cast(h_out.data_ptr() + 32 * off), err, 256) != 0:
                    raise RuntimeError(err.value)
                off += 1 << Lg
            return res

        t0 = time.perf_counter()
        res = host_loop()
        per_call_e2e_ms = (time.perf_counter() - t0) * 1e3
        exact = exact and b"".join(res) == self.graph_msm and bool(torch.equal(h_out, self.graph_ntt.cpu()))
        # the graph replay itself, host-timed the same way (launch + synchronize)
        t0 = time.perf_counter()
        b.batch_plan_launch(self.plan, s)
        torch.cuda.synchronize()
        graph_wall_ms = (time.perf_counter() - t0) * 1e3
        return {"per_call": {"device_resident_loop_ms": per_call_ms, "host_buffer_loop_ms": per_call_e2e_ms,
                             "graph_replay_wall_ms": graph_wall_ms, "bit_exact_with_graph": exact,
                             "calls_per_batch": len(self.sizes) + len(self.logs),
                             "note": "wall clock around each loop; every per-call form returns its result to "
                                     "the host, the graph form waits once"}}

    def e2e_step(self, dv, b):
        err = ctypes.create_string_buffer(256)
        cast = lambda t: ctypes.cast(ctypes.c_void_p(t.data_ptr()), ctypes.c_char_p)
        rc = dv.lib().dvgpu_batch_plan_run(b.handle, self.plan, self.h_scalars.data_ptr(), self.h_ntt.data_ptr(),
                                           cast(self.h_msm_out), cast(self.h_ntt_out), err, 256)
        if rc != 0:
            raise RuntimeError(err.value)
        return None

    def e2e_bytes(self):
        return 32 * (self.total + self.ntt_elems), 64 * len(self.sizes) + 32 * self.ntt_elems

    def roofline(self, tl, imad_peak, step_ms):
        macs = batch_macs(self.sizes, self.logs)
        ach = macs / (step_ms * 1e-3) / 1e12
        return ({"bound": "imad", "kernel": "whole batch graph (MSM accumulation dominant)", "achieved": ach,
                 "peak": imad_peak / 1e12, "unit": "TMAC/s", "frac": ach / (imad_peak / 1e12),
                 "algorithmic_macs_per_launch": macs, "launch_ms": step_ms}, None)

    def cpu(self, oracle, threads):
        ms, sample = batch_cpu(oracle, threads, self.h_points.numpy().tobytes(), self.sizes, self.logs,
                               self.h_scalars.numpy().tobytes(), self.h_ntt.numpy().tobytes())
        return None, ms, sample


R_MOD = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001


def fr_sub_bytes(a: bytes, b: bytes) -> bytes:
    """subtract_polynomials (crates/protocol/src/domain.rs:169-179) on
    canonical Fr coefficient bytes, vectorised: limb-wise borrow chain, + r
    where negative, trimmed."""
    import numpy as np
    n = max(len(a), len(b), 32) // 32
    x = np.zeros((n, 4), dtype=np.uint64)
    y = np.zeros((n, 4), dtype=np.uint64)
    x[:len(a) // 32] = np.frombuffer(a, dtype=np.uint64).reshape(-1, 4)
    y[:len(b) // 32] = np.frombuffer(b, dtype=np.uint64).reshape(-1, 4)
    r = np.array([(R_MOD >> (64 * i)) & (2**64 - 1) for i in range(4)], dtype=np.uint64)
    out = np.zeros_like(x)
    borrow = np.zeros(n, dtype=np.uint64)
    for i in range(4):
        t = x[:, i] - y[:, i]
        b1 = (x[:, i] < y[:, i]).astype(np.uint64)
        out[:, i] = t - borrow
        borrow = b1 | ((t < borrow).astype(np.uint64))
    neg = borrow == 1
    carry = np.zeros(n, dtype=np.uint64)
    for i in range(4):
        t = out[:, i] + r[i]
        c1 = (t < out[:, i]).astype(np.uint64)
        s_ = t + carry
        carry = c1 | (s_ < t).astype(np.uint64)
        out[:, i] = np.where(neg, s_, out[:, i])
    raw = out.tobytes()
    k = n
    while k > 1 and not any(raw[32 * (k - 1):32 * k]):
        k -= 1
    return raw[:32 * k]


def poly_work_fme(a):
    """Fr multiplications of one sparse-update polynomial step in the flat
    kernels of poly.cu: vanishing values N a and derivatives a^2 at tree
    creation; Cauchy pair sums 1 + 2R products per pair for R rows sharing
    the den chain (one call of 1 row, one of 3); power sums a^2 per
    interpolation row (9 rows); N = next_pow2(a).  Transforms, inversions,
    additions and shuffles are not counted."""
    big_n = max(2, 1 << (a - 1).bit_length())
    return big_n * a + a * a + 3 * a * a + 7 * a * a + 9 * a * a


class PolyOp:
    """The field work of one sparse update over an affected set of a points
    (crates/protocol/src/dynaverse/sparse.rs:125-236): subproduct tree,
    Cauchy weights, nine interpolations (anchor/changed/zero-quotient locals
    of the three multiplication wires), three Cauchy sums, the product
    updated_0 updated_1 and its exact division by the vanishing polynomial.
    Values are seeded uniform Fr; the third wire's values are the products of
    the first two at the points, so the division is exact as in the
    reference."""

    def __init__(self, args):
        self.a = 1 << args.log_n
        self.metric = f"sparse-update polynomial work a={self.a} ms"
        self.workload = (f"SubproductTree over {self.a} points + Cauchy weights + 9 interpolations + 3 Cauchy "
                         f"sums + product + exact division by the vanishing polynomial")
        self.profile = f"poly_sparse_update_{self.a}"

    def setup(self, torch, b, s, rank):
        from oracle import oracle
        a = self.a
        self.points = oracle.uniform_fr(9100 + rank, a)
        u0 = oracle.uniform_fr(9101, a)
        u1 = oracle.uniform_fr(9102, a)
        w = lambda buf, i: int.from_bytes(buf[32 * i:32 * i + 32], "little")
        u2 = b"".join((w(u0, i) * w(u1, i) % R_MOD).to_bytes(32, "little") for i in range(a))
        self.values9 = u0 + u1 + u2 + b"".join(oracle.uniform_fr(9110 + r, a) for r in range(6))
        self.weighted3 = b"".join(oracle.uniform_fr(9120 + r, a) for r in range(3))
        self.tune_log = None
        self.config = {"points": a, "interpolation_rows": 9, "cauchy_rows": 4}
        self.h2d = 32 * (a + 9 * a + 3 * a + a) + 0
        self.d2h = 0

    def run(self, b):
        import hashlib
        t = b.tree_create(self.points)
        try:
            weights = t.inverse_derivatives()
            cauchy_weights = t.cauchy_sums(weights)
            polys = t.interpolate(self.values9, 9)
            cauchy_values = t.cauchy_sums(self.weighted3, 3)
            product = b.poly_multiply(polys[0], polys[1])
            quotient = b.poly_divide_exact(fr_sub_bytes(product, polys[2]), t.vanishing())
        finally:
            t.close()
        self.last = (weights, cauchy_weights, polys, cauchy_values, quotient)
        h = hashlib.sha256()
        for part in (weights, cauchy_weights, b"".join(polys), cauchy_values, quotient):
            h.update(part)
        return h.hexdigest()

    def step(self, b, s):
        return self.run(b)

    def host_inputs(self, torch):
        pass

    def e2e_step(self, dv, b):
        return self.run(b)

    def e2e_bytes(self):
        a = self.a
        # H2D: points, weights (cauchy), 9 value rows, 3 weight rows, two product
        # operands, numerator and divisor; D2H: every returned vector
        h2d = 32 * (a + a + 9 * a + 3 * a + 2 * a + 3 * a + (a + 1))
        d2h = 32 * (a + a + 9 * a + 3 * a + 2 * a + (a + 1) + a)
        return h2d, d2h

    def roofline(self, tl, imad_peak, step_ms):
        macs = poly_work_fme(self.a) * 136
        ach = macs / (step_ms * 1e-3) / 1e12
        return ({"bound": "imad", "kernel": "whole step (k_powsum power sums and k_fracsum pair sums dominant)", "achieved": ach,
                 "peak": imad_peak / 1e12, "unit": "TMAC/s", "frac": ach / (imad_peak / 1e12),
                 "algorithmic_macs_per_launch": macs, "launch_ms": step_ms}, None)

    def cpu(self, oracle, threads):
        t0 = time.perf_counter()
        out = poly_cpu(oracle, self.points, self.values9, self.weighted3)
        ms = (time.perf_counter() - t0) * 1e3
        agree = out == self.last if hasattr(self, "last") else None
        return None, ms, (f"one full step (a={self.a}) through the oracle's restatement of "
                          f"domain/fast.rs, 1 thread; identical to the GPU's: {agree}")


def poly_cpu(oracle, points, values9, weighted3):
    a = len(points) // 32
    with oracle.Tree(points) as t:
        weights = t.inverse_derivatives()
        cauchy_weights = t.cauchy_sums(weights)
        polys = [t.interpolate(values9[32 * a * r:32 * a * (r + 1)]) for r in range(9)]
        cauchy_values = b"".join(t.cauchy_sums(weighted3[32 * a * r:32 * a * (r + 1)]) for r in range(3))
        product = oracle.poly_mul(polys[0], polys[1])
        quotient = oracle.poly_div_exact(fr_sub_bytes(product, polys[2]), t.vanishing())
    return weights, cauchy_weights, polys, cauchy_values, quotient


def pairing_fme(equations, terms_per_eq, distinct_g2, per_equation):
    """Fq multiplications of the lane-group pairing as implemented, all six
    lanes of a group counted: an Fq12 product is a three-term Karatsuba over
    Fq4, 18 Fq2 products (54 Fq-mul); a square the same with Fq4 squares, 18
    Fq2 squares (36); a cyclotomic square 12 Fq2 squares (24); a sparse line
    product 18 Fq2 products (54); the product of two lines 6 Fq2 products
    (18); scaling a line by its P 4 Fq-mul.  Each distinct G2 point is
    prepared once: 65 doublings and 23 additions whose Fq2 products are
    spread over the group (13 and 16 per step, 3 Fq-mul each).  The Miller
    loops, 65 squares and 88 line steps: one per term (per_equation false;
    the terms' values then meet in one product each), or the multi-Miller
    loop of two-term equations (per_equation true: one square per step, both
    lines scaled, multiplied together and into f by one product).  Per
    equation: the easy part (an Fq6 inverse, counted once although every
    lane of the group repeats it: 37 Fq-mul and an Fq inverse by divsteps,
    integer work counted as its one closing Montgomery product; four
    products, two of them inside the inverse, and a q^2 Frobenius); three
    exponentiations by z over its width-4 NAF
    (63 cyclotomic squares and 16 products each); and the hard part's 13
    products, 8 cyclotomic squares and three Frobenius maps
    (18 + 12 + 30)."""
    prep = 65 * 13 * 3 + 23 * 16 * 3
    if per_equation:
        assert terms_per_eq == 2
        miller = 65 * 36 + 88 * (8 + 18 + 54)
    else:
        miller = terms_per_eq * (65 * 36 + 88 * (4 + 54)) + (terms_per_eq - 1) * 54
    easy = (37 + 1) + 4 * 54 + 12
    hard = 3 * (63 * 24 + 16 * 54) + 13 * 54 + 8 * 24 + (18 + 12 + 30)
    return distinct_g2 * prep + equations * (miller + easy + hard)


class PairingOp:
    """Pairing-product checks in the shape of the rebuild's cache checks
    (PairingChecks::equal_prepared, crates/protocol/src/verification.rs
    :55-77): every equation is e(L_i, G) = e(R_i, D) for the fixed G2
    generator G and a fixed divisor D = [d]G2, moved to one side as
    e(L_i, G) e(-R_i, D) = 1, with L_i = [a_i]G1 and R_i = [a_i / d]G1; one
    final exponentiation per equation; every third equation has R_i off by one
    multiple of G1, so a third of the verdicts are false.  The two G2 points
    are prepared once per call."""

    def __init__(self, args):
        self.eqs = 1 << args.log_n
        self.metric = f"pairing checks, {self.eqs} equations x 2 terms, ms"
        self.workload = (f"{self.eqs} BN254 cache-check equations e(L_i, G) e(-R_i, D) = 1 over a fixed generator G "
                         f"and divisor D (one in three broken): Miller loops + one final exponentiation each")
        self.profile = f"pairing_check_{self.eqs}"

    def setup(self, torch, b, s, rank):
        from oracle import oracle
        n = self.eqs
        sa = oracle.uniform_fr(6100 + rank, n)
        d = int.from_bytes(oracle.uniform_fr(6200 + rank, 1), "little")
        d_inv = pow(d, R_MOD - 2, R_MOD)
        a = [int.from_bytes(sa[32 * i:32 * i + 32], "little") for i in range(n)]
        r = b"".join(((x * d_inv + (k % 3 == 1)) % R_MOD).to_bytes(32, "little") for k, x in enumerate(a))
        q_mod = 0x30644E72E131A029B85045B68181585D97816A916871CA8D3C208C16D87CFD47
        pl, pr = oracle.fixed_base_g1(sa), oracle.fixed_base_g1(r)
        gen2 = oracle.fixed_base_g2((1).to_bytes(32, "little"))
        div2 = oracle.fixed_base_g2(d.to_bytes(32, "little"))
        neg = lambda p: p[:32] + ((q_mod - int.from_bytes(p[32:], "little")) % q_mod).to_bytes(32, "little")
        self.g1 = b"".join(pl[64 * i:64 * i + 64] + neg(pr[64 * i:64 * i + 64]) for i in range(n))
        self.g2 = (gen2 + div2) * n
        self.offsets = list(range(0, 2 * n + 1, 2))
        self.qidx = [0, 1] * n
        # G and D prepared once, as the rebuild's tables hold them (setup, not timed)
        self.prepared = b.g2_prepare(gen2 + div2) if b is not None else None
        self.tune_log = None
        self.config = {"equations": n, "terms_per_equation": 2, "distinct_g2": 2,
                       "g2_prepared": "once, in setup (dvgpu_bn254_g2_prepare)"}

    def run(self, b):
        return tuple(b.pairing_check_prepared(self.g1, self.prepared, self.qidx, self.offsets))

    def step(self, b, s):
        return self.run(b)

    def host_inputs(self, torch):
        pass

    def e2e_step(self, dv, b):
        return self.run(b)

    def e2e_bytes(self):
        return len(self.g1) + len(self.g2) + 8 * len(self.offsets), self.eqs

    def per_equation(self, torch):
        """Whether the library runs the multi-Miller loop for this batch: more
        terms than one wave of per-term groups (k_miller_multi at 206
        registers holds 2 blocks of 20 groups per SM)."""
        return 2 * self.eqs > torch.cuda.get_device_properties(0).multi_processor_count * 2 * 20

    def roofline(self, tl, imad_peak, step_ms):
        import torch
        per_eq = self.per_equation(torch)
        macs = pairing_fme(self.eqs, 2, 0, per_eq) * 136
        ach = macs / (step_ms * 1e-3) / 1e12
        kernel = "k_miller_multi (%s) + k_final_exp (whole call)" % ("a group per equation" if per_eq
                                                                       else "a group per term")
        return ({"bound": "imad", "kernel": kernel, "achieved": ach,
                 "peak": imad_peak / 1e12, "unit": "TMAC/s", "frac": ach / (imad_peak / 1e12),
                 "algorithmic_macs_per_launch": macs, "launch_ms": step_ms}, None)

    def extra(self, torch, dv, b, s):
        one = (self.g1[:128], self.prepared, [0, 1], [0, 2])
        b.pairing_check_prepared(*one)
        t0 = time.perf_counter()
        for _ in range(5):
            b.pairing_check_prepared(*one)
        single = (time.perf_counter() - t0) * 1e3 / 5
        t0 = time.perf_counter()
        plain = b.pairing_check(self.g1, self.g2, self.offsets)
        unprepared = (time.perf_counter() - t0) * 1e3
        return {"single_equation_ms": single,
                "unprepared_call_ms": unprepared,
                "unprepared_call_note": "the same equations through dvgpu_bn254_pairing_check, which prepares "
                                        "the two G2 points inside the call",
                "unprepared_same_verdicts": tuple(plain) == self.run(b)}

    def cpu(self, oracle, threads):
        k = min(self.eqs, 32 * threads)
        t0 = time.perf_counter()
        out = oracle.pairing_check(self.g1[:128 * k], self.g2[:256 * k], self.offsets[:k + 1], threads=threads)
        ms = (time.perf_counter() - t0) * 1e3
        return None, ms * self.eqs / k, (f"{k} equations on {threads} threads, scaled to {self.eqs}; "
                                         f"verdicts identical to the GPU's: {out == list(self.run(self._b))[:k]}")


def make_op(args):
    return {"msm": lambda: MsmOp(args), "msmres": lambda: ResidentMsmOp(args), "g2msm": lambda: MsmOp(args, g2=True),
            "ntt": lambda: NttOp(args), "sparse": lambda: SparseOp(args), "fixedbase": lambda: FixedBaseOp(args),
            "batch": lambda: BatchOp(args), "g2check": lambda: G2CheckOp(args), "serve": lambda: ServeOp(args),
            "proofs": lambda: ProofServeOp(args),
            "ecntt": lambda: EcNttOp(args), "poly": lambda: PolyOp(args), "pairing": lambda: PairingOp(args)}[args.op]()


# ----------------------------------------------------------------- reference arm
def run_reference(args, rank, world):
    """--impl reference: the CPU implementation of the path on host cores."""
    if rank != 0:
        return
    from oracle import oracle
    threads = os.cpu_count() or 1
    op = args.op
    n = 1 << args.log_n
    if op == "proofs":
        p = ProofServeOp(args)
        p._inputs()
        cpu = ProofsCpu(p, threads)
        cpu.sample(2.0)  # warm-up
        steps = max(1, args.steps)
        rates = [r for r in (cpu.sample(30.0 / steps) for _ in range(steps)) if r is not None]
        value = sum(rates) / len(rates) if rates else None
        print(json.dumps({"impl": "reference", "metric": p.metric, "value": value, "unit": "proofs/s",
                          "n_gpus": world, "steps": steps, "warmup": args.warmup, "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "u64 limbs (Fq/Fr, exact)",
                          "data": "synthetic (seeded trapdoors, uniform valid witnesses, seeded update stream)",
                          "config": p.config(1),
                          "cpu_baseline": {"value": value, "unit": "proofs/s", "cores": threads, "kind": "port",
                                           "sample": cpu.describe()},
                          "e2e": {"value": value, "unit": "proofs/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0},
                          "note": ("reference = the oracle's restatement of the reference's update-proof steps "
                                   "(oracle/dynaverse.py over oracle/bn254_oracle.cpp); the reference's own "
                                   "Rust/arkworks code cannot be built in this image")}), flush=True)
        return
    if op in ("msm", "msmres", "g2msm"):
        g2 = op == "g2msm"
        tau = oracle.uniform_fr(2812, 1)
        fb = oracle.fixed_base_g2 if g2 else oracle.fixed_base_g1
        points = fb(oracle.fr_powers(tau, n), threads=threads)
        scalars = oracle.uniform_fr(2813, n)
        fn = (lambda: (oracle.msm_g2 if g2 else oracle.msm_g1)(points, scalars, threads=threads))
        metric = f"{'G2' if g2 else 'G1'} MSM 2^{args.log_n} ms"
        sample = f"full 2^{args.log_n}-point MSMs, window-parallel Pippenger"
    elif op == "ntt":
        vals = oracle.uniform_fr(3000, n)
        fn = lambda: oracle.ntt(vals, args.kind)
        metric = f"Fr NTT 2^{args.log_n} ms ({args.kind})"
        sample = f"full 2^{args.log_n} transforms, 1 thread (radix-2)"
        threads = 1
    elif op == "sparse":
        import numpy as np
        bases = oracle.fixed_base_g1(oracle.fr_powers(oracle.uniform_fr(2812, 1), n), threads=threads)
        idx = np.random.default_rng(5150).choice(n, size=args.k, replace=False).astype(np.uint64)
        vals = oracle.uniform_fr(5151, args.k)
        fn = lambda: oracle.sparse_msm_g1(bases, idx, vals, threads=threads)
        metric = f"sparse G1 MSM k={args.k} over 2^{args.log_n} bases us"
        sample = f"k={args.k} sparse MSMs"
    elif op == "ecntt":
        rows = min(args.rows, threads)
        pts = oracle.fixed_base_g1(oracle.uniform_fr(8100, rows << args.log_n), threads=threads)
        fn = lambda: oracle.g1_fft(pts, 1 << args.log_n, False, threads=threads)
        metric = EcNttOp(args).metric
        sample = f"{rows}-row G1 transforms of 2^{args.log_n} points on {rows} threads, scaled to {args.rows} rows"
        ecntt_scale = args.rows / rows
    elif op == "serve":
        sizes = ServeOp.SIZES
        stream = serve_stream(sizes, 400)
        used = sorted(set(j for j, _ in stream))
        bases = {j: oracle.fixed_base_g1(oracle.fr_powers(oracle.uniform_fr(7000 + j, 1), sizes[j]), threads=threads)
                 for j in used}
        vals = [oracle.uniform_fr(7300 + t, len(idx)) for t, (_, idx) in enumerate(stream)]

        def fn():
            for (j, idx), v in zip(stream, vals):
                oracle.sparse_msm_g1(bases[j], idx, v, threads=threads)

        metric = ServeOp(args).metric
        sample = "passes over the first 400 requests of the update stream (sparse delta MSMs)"
    elif op == "batch":
        sizes, logs = batch_workload(BatchOp.LOG_BASES)
        nb = 1 << BatchOp.LOG_BASES
        bases = oracle.fixed_base_g1(oracle.fr_powers(oracle.uniform_fr(2812, 1), nb), threads=threads)
        scalars = oracle.uniform_fr(2813, min(sum(sizes), (1 << 20) + nb))
        ntt_vals = oracle.uniform_fr(3000, sum(1 << L for L in logs[:8]))
        est = []

        def fn():
            ms, smp = batch_cpu(oracle, threads, bases, sizes, logs, scalars, ntt_vals)
            est.append((ms, smp))

        metric = BatchOp(args).metric
        sample = "batch estimates"
    elif op == "g2check":
        gop = G2CheckOp(args)
        k = min(n, 1 << 13)
        wire = (oracle.fixed_base_g2(oracle.uniform_fr(2900, k // 2), threads=threads) +
                oracle.g2_twist_points(2901, k - k // 2))
        fn = lambda: oracle.g2_check(wire, gop.alg, threads=threads)
        metric = gop.metric
        sample = f"{k}-point checks (half [s]G2, half twist points) on {threads} threads, scaled to 2^{args.log_n}"
        g2check_scale = n / k
    elif op == "pairing":
        pop = PairingOp(args)
        pop.setup(None, None, None, 0)
        k = min(pop.eqs, 32 * threads)
        fn = lambda: oracle.pairing_check(pop.g1[:128 * k], pop.g2[:256 * k], pop.offsets[:k + 1], threads=threads)
        metric = pop.metric
        sample = f"{k}-equation checks on {threads} threads, scaled to {pop.eqs} equations"
        pairing_scale = pop.eqs / k
    elif op == "poly":
        pop = PolyOp(args)

        class _B:  # setup needs no device
            pass
        pop.setup(None, _B(), None, 0)
        fn = lambda: poly_cpu(oracle, pop.points, pop.values9, pop.weighted3)
        metric = pop.metric
        sample = f"full sparse-update polynomial steps (a={pop.a}) through domain/fast.rs restated, 1 thread"
        threads = 1
    else:
        sc = oracle.fr_powers(oracle.uniform_fr(2812, 1), n)
        fn = lambda: oracle.fixed_base_g1(sc, threads=threads)
        metric = f"fixed-base G1 2^{args.log_n} ms"
        sample = f"full 2^{args.log_n}-point fixed-base generations"
    ours = make_op(args)  # the GPU arm's metric and workload, for the same line shape
    metric = ours.metric
    t0 = time.perf_counter()
    fn()
    first = (time.perf_counter() - t0) * 1e3
    steps = max(1, min(args.steps, int(90e3 // max(first, 1.0))))
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        fn()
        times.append((time.perf_counter() - t0) * 1e3)
    value = sum(times) / len(times)
    if op == "batch":
        value = sum(e[0] for e in est[1:]) / len(est[1:])
        sample = f"batch estimates, each from {est[-1][1]}"
    if op == "ecntt":
        value *= ecntt_scale
    if op == "pairing":
        value *= pairing_scale
    if op == "g2check":
        value *= g2check_scale
    higher = False
    ms_step = value
    if op == "serve":
        value = len(stream) / (value / 1e3)  # updates per second
        higher = True
    if op == "sparse":
        value *= 1e3  # us
    unit = "us" if op == "sparse" else ("updates/s" if op == "serve" else "ms")
    line = {
        "impl": "reference", "metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": higher,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64 limbs (Fq/Fr, exact)", "data": "synthetic",
        "config": {"workload": ours.workload, "op": op, "parallelism": "host threads"},
        "cpu_baseline": {"value": value, "unit": unit, "cores": threads, "kind": "port",
                         "sample": f"{steps} {sample} (after 1 warm-up)"},
        "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": ("reference = C++ restatement of arkworks 0.4 semantics (oracle/); the reference's own "
                 "Rust/arkworks/ICICLE code cannot be built in this image"),
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------- our arm
def max_over_ranks(ms, world, device="cuda"):
    """The slowest rank's time (every rank calls this at the same point)."""
    if world <= 1:
        return ms
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rates(total_ms, steps, world):
    """N independent replicas (nothing is sharded): per-step time of the
    slowest rank, and the whole-job time per unit of work = that / N."""
    return total_ms / steps, total_ms / (steps * world)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import torch
    import torch.distributed as dist
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    from __graft_entry__ import load_package
    dv = load_package()
    b = dv.DvgpuBackend()
    # a dedicated stream: every entry point gets its handle (a null handle
    # would select the owner's own stream), so the events below bracket the
    # work itself, including graph replays that return before completion
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    s = stream.cuda_stream
    op = make_op(args)
    op._b = b
    if args.probe:
        proof_probe(dv, args.probe, 1 << args.log_n)
        b.close()
        return
    if hasattr(op, "run_standalone"):
        try:
            bus = torch.cuda.get_device_properties(dev).pci_bus_id
        except AttributeError:
            bus = None
        sampler = ClockSampler(bus if isinstance(bus, str) else None)
        line = op.run_standalone(args, torch, dv, b, s, sampler, b.probe_imad_rate, world)
        if rank == 0:
            print(json.dumps(line), flush=True)
        b.close()
        if world > 1:
            dist.destroy_process_group()
        return
    op.setup(torch, b, s, rank)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    result = None
    for _ in range(args.warmup):
        result = op.step(b, s)
    torch.cuda.synchronize()

    try:
        bus = torch.cuda.get_device_properties(dev).pci_bus_id
    except AttributeError:
        bus = None
    sampler = ClockSampler(bus if isinstance(bus, str) else None)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    launches0 = b.launch_count()
    b.msm_timeline(True)
    step_ms = []
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = op.step(b, s)
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        if r != result:
            raise RuntimeError("result changed between steps")
    torch.cuda.synchronize()
    tl = b.msm_timeline(False)
    launches = b.launch_count() - launches0 + getattr(op, "launches_per_step", 0) * args.steps
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    total_ms = max_over_ranks(sum(step_ms), world)
    ms_per_step, value = replica_rates(total_ms, args.steps, world)

    # ---- end to end through the C-ABI with pinned host buffers
    op.host_inputs(torch)
    torch.cuda.synchronize()
    r0 = op.e2e_step(dv, b)
    if result is not None and r0 != result:
        raise RuntimeError("host-buffer call differs from the device-resident call")
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        op.e2e_step(dv, b)
    e2e_total = max_over_ranks((time.perf_counter() - t0) * 1e3, world)
    e2e_ms = replica_rates(e2e_total, args.e2e_steps, world)[1]

    extra = op.extra(torch, dv, b, s) if hasattr(op, "extra") else {}
    imad_peak = b.probe_imad_rate()
    roof, whole = op.roofline(tl, imad_peak, ms_per_step)
    roof["traffic"] = load_traffic(op.profile)
    roof["peak_source"] = "dvgpu_probe_imad_rate in this run (madc.lo/hi chains on all SMs)"
    scale = 1e3 if args.op == "sparse" else 1.0  # sparse reported in microseconds
    unit = "us" if args.op == "sparse" else "ms"
    h2d, d2h = op.e2e_bytes()
    config = {"workload": op.workload, "op": args.op,
              "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
              "l2": "flushed between steps (256 MB write)"}
    config.update(op.config)
    line = {
        "metric": op.metric, "value": value * scale, "unit": unit, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32 limbs (Fq/Fr Montgomery, exact)", "data": "synthetic",
        "config": config,
        "e2e": {"value": e2e_ms * scale, "unit": unit, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "call": "reference-facing C-ABI entry point with pinned host buffers"},
        "roofline": roof,
        "gpu_launches": launches,
        "clocks": clocks,
    }
    if whole:
        line[getattr(op, "secondary_key", "msm_roofline")] = whole
    line.update(extra)
    if tl.calls:
        line["phases_ms"] = {name: tl.ms[k] / tl.calls for k, name in enumerate(dv.MSM_PHASE_NAMES)}
    if op.tune_log:
        line["autotune"] = op.tune_log
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle
        threads = os.cpu_count() or 1
        cpu_out, cpu_ms, sample = op.cpu(oracle, threads)
        line["cpu_baseline"] = {"value": cpu_ms * scale, "unit": unit,
                                "cores": 1 if args.op in ("ntt", "poly") else threads, "kind": "port", "sample": sample}
        if cpu_out is not None:
            line["cpu_baseline"]["matches_gpu"] = cpu_out == result
    if rank == 0:
        print(json.dumps(line), flush=True)
    b.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
