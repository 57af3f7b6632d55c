"""CPU-only checks of the boundary: the C-ABI library loads, exports every
symbol include/dynaverse_gpu.h declares, and the field constants embedded in
the CUDA sources equal the values computed here with Python integers."""
import ctypes
import os
import re
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import bn254_py as b  # noqa: E402

HEADER = os.path.join(ROOT, "include", "dynaverse_gpu.h")
CSRC = os.path.join(ROOT, "zkp-dynaverse_b200", "csrc")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dvgpu_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_reference_entry_points():
    names = set(declared_functions())
    # the entry points the reference's Rust crate binds (icicle.rs:35-57,
    # setup.rs:47-52, g2_validation.rs:84-93)
    for n in ["dvgpu_backend_create", "dvgpu_backend_create_with_large_bucket_factor", "dvgpu_backend_destroy",
              "dvgpu_backend_device_identity", "dvgpu_backend_batch_stats", "dvgpu_backend_memory_info",
              "dvgpu_bn254_msm", "dvgpu_bn254_msm_batch", "dvgpu_bn254_g2_msm", "dvgpu_bn254_ntt",
              "dvgpu_bn254_msm_profiled", "dvgpu_bn254_fixed_base", "dvgpu_setup_mode", "dvgpu_setup_stats",
              "dvgpu_bn254_g2_validation_inspect", "dvgpu_g2_validation_stats", "dvgpu_g2_validation_traffic",
              "dvgpu_bn254_fixed_base_g2_checked", "dvgpu_reserve_batch",
              # diagnostics bound by icicle.rs:54, g2_validation.rs:91-94, resident_profile.rs:40
              "dvgpu_bn254_msm_timeline", "dvgpu_g2_kernel_config_set", "dvgpu_g2_kernel_config_get",
              "dvgpu_g2_kernel_resources", "dvgpu_g2_experiment_stats", "dvgpu_resident_call_profiled"]:
        assert n in names, n


def test_diagnostic_struct_layouts(dv, tmp_path):
    """The byte layouts the reference's Rust bindings assert
    (crates/gpu/src/g2_validation.rs:48-49) and the timeline / profile
    records, in C and in the Python mirror."""
    src = tmp_path / "sizes.c"
    src.write_text('#include "dynaverse_gpu.h"\n'
                   "_Static_assert(sizeof(DvgpuG2KernelConfig) == 16, \"config\");\n"
                   "_Static_assert(sizeof(DvgpuG2KernelResources) == 56, \"resources\");\n"
                   "_Static_assert(sizeof(DvgpuG2ExperimentStats) == 24, \"experiment\");\n"
                   "_Static_assert(sizeof(DvgpuMsmTimeline) == 8 * (5 * 9 + 2 * 10 + 6), \"timeline\");\n"
                   "_Static_assert(sizeof(DvgpuResidentProfile) == 96, \"profile\");\n")
    subprocess.run(["gcc", "-fsyntax-only", "-I", os.path.dirname(HEADER), str(src)], check=True)
    assert ctypes.sizeof(dv.G2KernelConfig) == 16 and ctypes.sizeof(dv.G2KernelResources) == 56
    assert ctypes.sizeof(dv.G2ExperimentStats) == 24 and ctypes.sizeof(dv.ResidentProfile) == 96
    assert ctypes.sizeof(dv.MsmTimeline) == 8 * (5 * 9 + 2 * 10 + 6)


def test_dynaverse_struct_layouts(dv, tmp_path):
    """The update-proof engine's records agree in C and in the Python mirror."""
    src = tmp_path / "dv_sizes.c"
    stats = ctypes.sizeof(dv.DynaverseStats)
    info = ctypes.sizeof(dv.DynaverseParamsInfo)
    res = ctypes.sizeof(dv.DynaverseResult)
    src.write_text('#include "dynaverse_gpu.h"\n'
                   f"_Static_assert(sizeof(DvgpuDynaverseStats) == {stats}, \"stats\");\n"
                   f"_Static_assert(sizeof(DvgpuDynaverseParamsInfo) == {info}, \"info\");\n"
                   f"_Static_assert(sizeof(DvgpuDynaverseResult) == {res}, \"result\");\n"
                   "_Static_assert(DVGPU_DYNAVERSE_PROOF_BYTES == 3968 + 5312 + 24, \"proof\");\n")
    subprocess.run(["gcc", "-fsyntax-only", "-I", os.path.dirname(HEADER), str(src)], check=True)
    assert stats == 8 * 23 and dv.DYNAVERSE_PROOF_BYTES == 9304


def test_every_symbol_the_reference_crate_binds_is_declared():
    """Every dvgpu_* function named in the reference's Rust extern blocks
    (crates/gpu/src) is declared, so the crate links against the library
    (the research probes among them return -1)."""
    bound = {"dvgpu_backend_create", "dvgpu_backend_create_with_large_bucket_factor", "dvgpu_backend_destroy",
             "dvgpu_backend_device_identity", "dvgpu_backend_memory_info", "dvgpu_backend_batch_stats",
             "dvgpu_bn254_msm", "dvgpu_bn254_msm_profiled", "dvgpu_bn254_msm_timeline", "dvgpu_bn254_msm_batch",
             "dvgpu_bn254_g2_msm", "dvgpu_bn254_ntt", "dvgpu_bn254_fixed_base", "dvgpu_setup_mode",
             "dvgpu_setup_stats", "dvgpu_reserve_batch", "dvgpu_bn254_g2_validation_inspect",
             "dvgpu_g2_validation_stats", "dvgpu_g2_validation_traffic", "dvgpu_bn254_fixed_base_g2_checked",
             "dvgpu_g2_kernel_config_set", "dvgpu_g2_kernel_config_get", "dvgpu_g2_kernel_resources",
             "dvgpu_g2_experiment_stats", "dvgpu_resident_configure", "dvgpu_resident_call",
             "dvgpu_resident_seal", "dvgpu_resident_commit", "dvgpu_resident_stats", "dvgpu_resident_diagnostics",
             "dvgpu_resident_call_profiled", "dvgpu_bn254_tower_inspect", "dvgpu_bn254_lines_inspect",
             "dvgpu_bn254_miller_inspect", "dvgpu_g2_psi_probe", "dvgpu_g2_test_corrupt_next"}
    assert not bound - set(declared_functions())


def test_research_probes_report_not_provided(dv):
    lib = dv.lib()
    err = ctypes.create_string_buffer(128)
    assert lib.dvgpu_bn254_miller_inspect(None, None, 0, None, 0, None, 0, None, 0, err, 128) == -1
    assert b"not provided" in err.value
    assert lib.dvgpu_g2_test_corrupt_next(None, 0) == -1


def test_diagnostics_reject_null_owner(dv):
    lib = dv.lib()
    cfg = dv.G2KernelConfig(128, 0, 0, 0)
    assert lib.dvgpu_g2_kernel_config_set(None, ctypes.byref(cfg)) == -1
    assert lib.dvgpu_g2_kernel_config_get(None, ctypes.byref(cfg)) == -1
    assert lib.dvgpu_g2_experiment_stats(None, ctypes.byref(dv.G2ExperimentStats())) == -1
    assert lib.dvgpu_g2_kernel_resources(None, 3, ctypes.byref(dv.G2KernelResources())) == -1
    prof = dv.ResidentProfile()
    assert lib.dvgpu_resident_call_profiled(None, None, None, ctypes.byref(prof), None, 0) == -1
    assert lib.dvgpu_bn254_msm_timeline(None, None, None, 0, None, None, None, None, None, 0) == -1


def test_library_exports_every_declared_symbol(dv):
    lib = dv.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_signatures_cover_header(dv):
    bound = {s[0] for s in dv.SIGNATURES}
    assert set(declared_functions()) <= bound


def _limbs32(v):
    return [(v >> (32 * i)) & 0xFFFFFFFF for i in range(8)]


def _cfg_values(text, cfg, prefix):
    body = text[text.index(f"struct {cfg}"):]
    body = body[:body.index("};")]
    vals = {}
    for name, val in re.findall(r"\b([A-Z0-9]+)\s*=\s*(0x[0-9a-fA-F]+)u", body):
        vals[name] = int(val, 16)
    return [vals[f"{prefix}{i}"] for i in range(8)], vals


@pytest.mark.parametrize("cfg,p", [("FqCfg", b.Q), ("FrCfg", b.R)])
def test_device_field_constants(cfg, p):
    text = open(os.path.join(CSRC, "field.cuh")).read()
    pl, vals = _cfg_values(text, cfg, "P")
    assert pl == _limbs32(p)
    assert vals["INV"] == (-pow(p, -1, 1 << 32)) % (1 << 32)
    one, _ = _cfg_values(text, cfg, "ONE")
    r2, _ = _cfg_values(text, cfg, "R2")
    assert one == _limbs32((1 << 256) % p)
    assert r2 == _limbs32((1 << 512) % p)


def _c_array(text, name):
    m = re.search(name + r"[^=]*=\s*\{(.*?)\};", text, flags=re.S)
    return [int(x, 16) for x in re.findall(r"0x[0-9a-fA-F]+", m.group(1))]


def _int_of(words):
    return sum(w << (32 * i) for i, w in enumerate(words))


def test_device_curve_and_psi_constants():
    g2 = open(os.path.join(CSRC, "g2.cu")).read()
    psi = _c_array(g2, "PSI_C")
    assert _int_of(psi[0:8]) == b.PSI_CX[0] and _int_of(psi[8:16]) == b.PSI_CX[1]
    assert _int_of(psi[16:24]) == b.PSI_CY[0] and _int_of(psi[24:32]) == b.PSI_CY[1]
    assert _int_of(_c_array(g2, "R_INT")) == b.R
    assert _int_of(_c_array(g2, "LAMBDA")) == 6 * b.BN_SEED ** 2
    assert _int_of(_c_array(g2, "SEED")) == b.BN_SEED
    gen = _c_array(g2, "G2_GEN")
    assert (_int_of(gen[0:8]), _int_of(gen[8:16])) == b.G2_GEN[0]
    assert (_int_of(gen[16:24]), _int_of(gen[24:32])) == b.G2_GEN[1]
    curve = open(os.path.join(CSRC, "curve.cuh")).read()
    body = curve[curve.index("Fq2 g2_b()"):]
    assert _int_of(_c_array(body, "c0")) == b.B2[0]
    assert _int_of(_c_array(body, "c1")) == b.B2[1]
    ntt = open(os.path.join(CSRC, "ntt.cu")).read()
    assert _int_of(_c_array(ntt, "ROOT28")) == b.root_of_unity(1 << 28)


def test_glv_constants_of_the_g1_transform():
    """beta/lambda of the G1 endomorphism and the lattice and rounding
    constants of the GLV split in ecntt.cu, derived here with Python integers
    (cube roots of unity matched on the generator; the short basis from the
    extended Euclidean algorithm on (r, lambda), Gallant-Lambert-Vanstone)."""
    import math
    src = open(os.path.join(CSRC, "ecntt.cu")).read()
    q, r = b.Q, b.R
    roots = lambda p: [pow(g, (p - 1) // 3, p) for g in range(2, 50) if pow(g, (p - 1) // 3, p) != 1][:1]
    w_q, w_r = roots(q)[0], roots(r)[0]
    pairs = [(be, la) for be in (w_q, w_q * w_q % q) for la in (w_r, w_r * w_r % r)
             if (be * b.G1_GEN[0] % q, b.G1_GEN[1]) == b.g1_mul(b.G1_GEN, la)]
    assert len(pairs) == 2  # (beta, lambda) and (beta^2, lambda^2)
    mine = [(be, la) for be, la in pairs if (be << 256) % q == _int_of(_c_array(src, "GLV_BETA"))]
    assert len(mine) == 1
    beta, lam = mine[0]
    r0, r1, t0, t1 = r, lam, 0, 1
    rs, ts = [r0, r1], [t0, t1]
    while r1:
        k = r0 // r1
        r0, r1, t0, t1 = r1, r0 - k * r1, t1, t0 - k * t1
        rs.append(r1)
        ts.append(t1)
    m = max(i for i in range(len(rs)) if rs[i] >= math.isqrt(r))
    a1, b1 = rs[m + 1], -ts[m + 1]
    a2, b2 = min([(rs[m], -ts[m]), (rs[m + 2], -ts[m + 2])], key=lambda v: v[0] ** 2 + v[1] ** 2)
    assert a1 * b2 - a2 * b1 == r
    g1 = ((b2 << 256) + r // 2) // r
    g2 = ((-b1 << 256) + r // 2) // r
    words = lambda name: int("".join(reversed(re.findall(r"0x([0-9a-f]+)ull",
                                                          re.search(name + r" = \{\{(.*?)\}\}", src).group(1)))), 16)
    assert int(re.search(r"GLV_A1 = (\d+)ull", src).group(1)) == a1 == b2
    assert words("GLV_B1ABS") == -b1 and words("GLV_A2") == a2
    assert words("GLV_G1") == g1 and words("GLV_G2") == g2
