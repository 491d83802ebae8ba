"""The C-ABI library loads and exports what include/beam_gpu.h declares; host
logic that needs no device. No compute calls run here."""
import ctypes
import os
import subprocess

import pytest

from conftest import ROOT


def test_library_exports_every_declared_symbol(beamlib):
    syms = beamlib.header_symbols()
    assert len(syms) >= 13
    L = beamlib.load()
    for s in syms:
        assert hasattr(L, s), s
    out = subprocess.run(["nm", "-D", "--defined-only", beamlib.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [s for s in syms if s not in exported]
    assert not missing, missing


def test_library_exports_only_the_c_abi(beamlib):
    out = subprocess.run(["nm", "-D", "--defined-only", beamlib.LIB_PATH], capture_output=True, text=True).stdout
    names = {line.split()[-1] for line in out.splitlines() if line.strip()}
    ours = {n for n in names if n.startswith("_ZN4beam")}
    assert not ours, sorted(ours)[:5]


def test_defaults_are_the_reference_constants(beamlib):
    L = beamlib.load()
    cfg = beamlib.Cfg()
    L.beam_cfg_default(ctypes.byref(cfg), 384, 51, 1, 1)
    # barbie.c:67-84
    assert (cfg.NN, cfg.Nmax, cfg.Nr, cfg.n_mtbin, cfg.LL) == (384, 100, 40, 5, 1.0)
    assert (cfg.UL_k1, cfg.LL_k1, cfg.BW_k1) == (51, 1, 1)
    assert cfg.precision == 0 and cfg.method == 0


def test_error_strings(beamlib):
    L = beamlib.load()
    for code in range(0, -10, -1):
        assert L.beam_gpu_strerror(code)
    assert L.beam_gpu_strerror(-12345) == b"unknown error"


def test_init_without_device_reports_enodev(beamlib):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    L = beamlib.load()
    h = ctypes.c_void_p()
    assert L.beam_gpu_init(0, ctypes.byref(h)) == beamlib.BEAM_ENODEV
    with pytest.raises(beamlib.BeamError):
        beamlib.Context(0)


def test_null_arguments_are_rejected(beamlib):
    L = beamlib.load()
    assert L.beam_gpu_init(0, None) == beamlib.BEAM_EINVAL
    assert L.beam_gpu_plan_create(None, None, None) == beamlib.BEAM_EINVAL
    assert L.beam_gpu_run(None, None, 0, None) == beamlib.BEAM_EINVAL
    assert L.beam_gpu_run_batch_ex(None, None, 0, None, 0) == beamlib.BEAM_EINVAL
    assert L.beam_gpu_plan_autotune(None, 0, None) == beamlib.BEAM_EINVAL
    assert L.beam_gpu_field_autotune(None, 64, None) == beamlib.BEAM_EINVAL
    d = ctypes.c_double
    assert L.beam_gpu_field_generate(None, 64, 1, d(0.56), d(0.5), d(1.0), None, 0, None) == beamlib.BEAM_EINVAL
    assert L.beam_gpu_field_launches(None) == -1


def test_server_host_side_argument_checks(beamlib):
    L = beamlib.load()
    beamlib._server_protos(L)
    cfg = beamlib.ServerCfg()
    L.beam_server_cfg_default(ctypes.byref(cfg))
    assert (cfg.mem_budget, cfg.max_active, cfg.max_plans) == (0, 4, 16)
    h = ctypes.c_void_p()
    assert L.beam_gpu_server_create(None, ctypes.byref(cfg), ctypes.byref(h)) == beamlib.BEAM_EINVAL
    job = ctypes.c_int64()
    assert L.beam_gpu_server_submit(None, None, None, ctypes.byref(job)) == beamlib.BEAM_EINVAL
    assert L.beam_gpu_server_wait(None, 1, 0, None) == beamlib.BEAM_EINVAL
    assert L.beam_gpu_server_take(None, 1, None) == beamlib.BEAM_EINVAL
    assert L.beam_gpu_server_memory(None, None, None) == beamlib.BEAM_EINVAL


def test_host_cli_usage_and_errors(tmp_path):
    exe = os.path.join(ROOT, "barbie_b200", "barbie")
    if not os.path.exists(exe):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "barbie_b200")], check=True)
    r = subprocess.run([exe, "64", "1"], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 1 and r.stdout.startswith("Usage:")  # barbie.c:58-60
    r = subprocess.run([exe, "64", "1", "11", "1", "1"], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 1 and "field_N64_R1.txt" in r.stderr
    (tmp_path / "field_N64_R1.txt").write_bytes(b"\0" * 80)
    r = subprocess.run([exe, "64", "1", "11", "1", "1"], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 1 and "expected" in r.stderr


def test_calpow_cli_usage_and_errors(tmp_path):
    exe = os.path.join(ROOT, "barbie_b200", "calpow_mom")
    if not os.path.exists(exe):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "barbie_b200")], check=True)
    r = subprocess.run([exe, "64"], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 1 and r.stdout.startswith("Usage:")  # calpow_mom.c:44-46
    r = subprocess.run([exe, "64", "1"], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 1 and "field_N64_R1.txt" in r.stderr
