"""Logging-layer parity (no GPU): rocsolver_log_* session rules and the bench / trace line
formats of the reference's logger (library/src/include/rocsolver_logger.hpp:171-205,
library/src/common/rocsolver_logger.cpp:177-330).  Calls here fail their argument checks
or return quickly, so nothing reaches a kernel launch; the reference logs an entry point
before its checks, so they are still logged."""
import ctypes
import os

import pytest

import rocsolver_b200 as rs

FAKE = ctypes.c_void_p(0x1000)


@pytest.fixture
def session(tmp_path, monkeypatch):
    logs = {k: tmp_path / f"{k}.log" for k in ("trace", "bench", "profile")}
    for k, p in logs.items():
        monkeypatch.setenv(f"ROCSOLVER_LOG_{k.upper()}_PATH", str(p))
    monkeypatch.setenv("ROCSOLVER_LAYER", "3")
    monkeypatch.setenv("ROCSOLVER_LEVELS", "2")
    assert rs.call("rocsolver_log_begin") == rs.SUCCESS
    yield logs
    rs.call("rocsolver_log_end")


def test_session_rules(monkeypatch):
    monkeypatch.delenv("ROCSOLVER_LAYER", raising=False)
    assert rs.call("rocsolver_log_end") == rs.INTERNAL_ERROR          # no session
    assert rs.call("rocsolver_log_set_layer_mode", 1) == rs.INTERNAL_ERROR
    assert rs.call("rocsolver_log_begin") == rs.SUCCESS
    assert rs.call("rocsolver_log_begin") == rs.INTERNAL_ERROR        # already open
    assert rs.call("rocsolver_log_set_max_levels", 0) == rs.INVALID_VALUE
    assert rs.call("rocsolver_log_set_max_levels", 3) == rs.SUCCESS
    assert rs.call("rocsolver_log_set_layer_mode", 7) == rs.SUCCESS
    assert rs.call("rocsolver_log_restore_defaults") == rs.SUCCESS
    assert rs.call("rocsolver_log_write_profile") == rs.SUCCESS
    assert rs.call("rocsolver_log_flush_profile") == rs.SUCCESS
    assert rs.call("rocsolver_log_end") == rs.SUCCESS
    monkeypatch.setenv("ROCSOLVER_LAYER", "not-a-number")
    assert rs.call("rocsolver_log_begin") == rs.INTERNAL_ERROR
    monkeypatch.setenv("ROCSOLVER_LAYER", "1")
    monkeypatch.setenv("ROCSOLVER_LEVELS", "0")
    assert rs.call("rocsolver_log_begin") == rs.INTERNAL_ERROR


def test_bench_and_trace_lines(session):
    h = rs.Handle()
    try:
        # invalid size: logged, then rejected before any launch
        st = rs.call("rocsolver_dgetrf_strided_batched", h.value, -1, 256, FAKE, 256, 65536,
                     FAKE, 256, FAKE, 2048)
        assert st == rs.INVALID_SIZE
        st = rs.call("rocsolver_sgetrs_strided_batched", h.value, rs.OP_T, 32, 4, FAKE, 32,
                     1024, FAKE, 32, FAKE, 32, 128, 0)
        assert st == rs.SUCCESS   # zero batch: quick return
        st = rs.call("rocsolver_dpotrf", h.value, rs.FILL_LOWER, -5, FAKE, 1, FAKE)
        assert st == rs.INVALID_SIZE
    finally:
        h.close()
    assert rs.call("rocsolver_log_end") == rs.SUCCESS
    bench = session["bench"].read_text().splitlines()
    trace = session["trace"].read_text()
    assert bench[0] == "ROCSOLVER LOG FILE"
    lines = [l for l in bench if l.startswith("./rocsolver-bench")]
    assert lines == [
        "./rocsolver-bench -f getrf_strided_batched -r d -m -1 -n 256 --lda 256 "
        "--strideA 65536 --strideP 256 --batch_count 2048",
        "./rocsolver-bench -f getrs_strided_batched -r s --trans T -n 32 --nrhs 4 --lda 32 "
        "--strideA 1024 --strideP 32 --ldb 32 --strideB 128 --batch_count 0",
        "./rocsolver-bench -f potrf -r d --uplo L -n -5 --lda 1",
    ]
    for name in ("rocsolver_dgetrf_strided_batched", "rocsolver_sgetrs_strided_batched",
                 "rocsolver_dpotrf"):
        assert f"------- ENTER {name} trace tree -------" in trace
        assert f"------- EXIT {name} trace tree -------" in trace
    # a second rocsolver_log_end has nothing to close
    assert rs.call("rocsolver_log_end") == rs.INTERNAL_ERROR


def test_disabled_by_default_writes_nothing(tmp_path, monkeypatch):
    p = tmp_path / "all.log"
    monkeypatch.setenv("ROCSOLVER_LOG_PATH", str(p))
    monkeypatch.delenv("ROCSOLVER_LAYER", raising=False)
    assert rs.call("rocsolver_log_begin") == rs.SUCCESS
    h = rs.Handle()
    try:
        rs.call("rocsolver_dgetrf_strided_batched", h.value, -1, 1, FAKE, 1, 1, FAKE, 1, FAKE, 1)
    finally:
        h.close()
    assert rs.call("rocsolver_log_end") == rs.SUCCESS
    text = p.read_text()
    assert "rocsolver-bench" not in text and "trace tree" not in text


@pytest.mark.gpu
def test_trace_kernels_and_profile_gpu(tmp_path, monkeypatch):
    """A real factor-and-solve under ROCSOLVER_LAYER = trace | profile | kernels and
    ROCSOLVER_LEVELS = 3: the trace tree holds the template-level step and its kernel
    launches, the profile counts them."""
    import numpy as np
    import torch
    path = tmp_path / "log.txt"
    monkeypatch.setenv("ROCSOLVER_LOG_PATH", str(path))
    monkeypatch.setenv("ROCSOLVER_LAYER", str(1 | 4 | 0x10))
    monkeypatch.setenv("ROCSOLVER_LEVELS", "3")
    assert rs.call("rocsolver_log_begin") == rs.SUCCESS
    h = rs.Handle(torch.cuda.current_stream().cuda_stream)
    try:
        n, bc = 64, 4
        A = torch.from_numpy(np.random.default_rng(0).uniform(-1, 1, (bc, n, n)) + 4 * np.eye(n)).cuda()
        P = torch.zeros(bc * n, dtype=torch.int32, device="cuda")
        I = torch.zeros(bc, dtype=torch.int32, device="cuda")
        B = torch.ones(bc, n, dtype=torch.float64, device="cuda")
        for _ in range(2):
            rs.check(rs.call("rocsolver_dgetrf_strided_batched", h.value, n, n, rs.ptr(A), n, n * n,
                             rs.ptr(P), n, rs.ptr(I), bc), "getrf")
        rs.check(rs.call("rocsolver_dgetrs_strided_batched", h.value, rs.OP_N, n, 1, rs.ptr(A), n,
                         n * n, rs.ptr(P), n, rs.ptr(B), n, n, bc), "getrs")
        torch.cuda.synchronize()
    finally:
        h.close()
    assert rs.call("rocsolver_log_end") == rs.SUCCESS
    text = path.read_text()
    assert "------- ENTER rocsolver_dgetrf_strided_batched trace tree -------" in text
    assert "rocsolver_getrf_template (m 64, n 64, lda 64, bc 4)" in text
    assert "    getrf_cta_kernel" in text
    assert "rocsolver_getrs_template (trans N, n 64, nrhs 1, lda 64, ldb 64, bc 4)" in text
    assert "------- PROFILE -------" in text
    assert "rocsolver_getrf_template: Calls: 2, Total Time:" in text
    assert "    getrf_cta_kernel: Calls: 2, Total Time:" in text


def test_complex_entry_points_log_their_precision(session):
    """The c / z entry points log with -r c / -r z, as the reference's do
    (rocsolver_logger.hpp get_precision for rocblas_float_complex / rocblas_double_complex),
    with conjugate-transpose solves logged as --trans C."""
    h = rs.Handle()
    try:
        st = rs.call("rocsolver_zgetrf_strided_batched", h.value, -1, 8, FAKE, 8, 64, FAKE, 8,
                     FAKE, 2)
        assert st == rs.INVALID_SIZE
        st = rs.call("rocsolver_cgetrs_strided_batched", h.value, rs.OP_C, 8, 1, FAKE, 8, 64,
                     FAKE, 8, FAKE, 8, 8, 0)
        assert st == rs.SUCCESS
        st = rs.call("rocsolver_zposv", h.value, rs.FILL_UPPER, -2, 1, FAKE, 1, FAKE, 1, FAKE)
        assert st == rs.INVALID_SIZE
    finally:
        h.close()
    assert rs.call("rocsolver_log_end") == rs.SUCCESS
    lines = [l for l in session["bench"].read_text().splitlines()
             if l.startswith("./rocsolver-bench")]
    assert lines[0].startswith("./rocsolver-bench -f getrf_strided_batched -r z -m -1 -n 8")
    assert lines[1].startswith("./rocsolver-bench -f getrs_strided_batched -r c --trans C")
    assert lines[2].startswith("./rocsolver-bench -f posv -r z --uplo U -n -2")
