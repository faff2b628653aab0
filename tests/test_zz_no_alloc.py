"""sap_blas_dots_noalloc: the dot products for callers that cannot allocate
device memory where they need the reduction (code under another framework's
caching allocator that owns the free memory, applications that budget GPU
memory once at start-up, loops in which cudaMalloc/cudaFree would
synchronise the device).  Called through the C ABI and checked against the
allocating entry point sap_blas_dots.  This file is collected last."""
import ctypes

import numpy as np
import pytest

import saplibrary_b200 as sap

LIMIT = 16_777_216  # vector length served by the fixed 64 KB scratch


def _call(fn, xs, ys, out, n):
    nq = len(xs)
    xa = (ctypes.c_void_p * nq)(*[t.data_ptr() for t in xs])
    ya = (ctypes.c_void_p * nq)(*[t.data_ptr() for t in ys])
    return fn(n, nq, xa, ya, ctypes.c_void_p(out.data_ptr()), None)


def test_rejects_lengths_beyond_the_scratch_limit():
    dummy = (ctypes.c_void_p * 1)(ctypes.c_void_p(16))
    rc = sap._lib.sap_blas_dots_noalloc(LIMIT + 1, 1, dummy, dummy, ctypes.c_void_p(16), None)
    assert rc == -100  # SAP_ERR_INVALID_ARGUMENT, nothing launched
    assert b"exceeds the fixed scratch limit" in sap._lib.sap_last_error()


@pytest.mark.gpu
@pytest.mark.parametrize("n,nq", [(1, 1), (4097, 2), (3_000_001, 4), (LIMIT, 1)])
def test_noalloc_matches_allocating_entry_point(n, nq):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(n + nq)
    xs = [torch.tensor(rng.standard_normal(n), device="cuda") for _ in range(nq)]
    ys = [torch.tensor(rng.standard_normal(n), device="cuda") for _ in range(nq)]
    ref = torch.empty(nq, device="cuda", dtype=torch.float64)
    assert _call(sap._lib.sap_blas_dots, xs, ys, ref, n) == 0
    torch.cuda.synchronize()
    outs = []
    for _ in range(2):  # two calls in a row share the same scratch
        out = torch.full((nq,), float("nan"), device="cuda", dtype=torch.float64)
        assert _call(sap._lib.sap_blas_dots_noalloc, xs, ys, out, n) == 0
        torch.cuda.synchronize()
        outs.append(out.cpu().numpy())
    for o in outs:
        assert np.allclose(o, ref.cpu().numpy(), rtol=1e-12, atol=1e-12)


def _other_processes_on_device(torch) -> bool:
    """True when NVML lists compute processes on the current device other
    than this one (their allocations change the device-wide free memory), or
    when NVML cannot tell.  The device is found by its PCI address, which
    does not depend on CUDA_VISIBLE_DEVICES."""
    import os
    try:
        import pynvml
        pr = torch.cuda.get_device_properties(torch.cuda.current_device())
        bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
        pynvml.nvmlInit()
        try:
            h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            procs = pynvml.nvmlDeviceGetComputeRunningProcesses(h)
            return any(p.pid != os.getpid() for p in procs)
        finally:
            pynvml.nvmlShutdown()
    except Exception:
        return True


@pytest.mark.gpu
def test_noalloc_allocates_no_device_memory():
    torch = pytest.importorskip("torch")
    n = 1_000_000
    x = torch.ones(n, device="cuda", dtype=torch.float64)
    out = torch.empty(1, device="cuda", dtype=torch.float64)
    assert _call(sap._lib.sap_blas_dots_noalloc, [x], [x], out, n) == 0  # first call: per-device set-up
    torch.cuda.synchronize()
    torch_bytes0 = torch.cuda.memory_allocated()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert _call(sap._lib.sap_blas_dots_noalloc, [x], [x], out, n) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert torch.cuda.memory_allocated() == torch_bytes0
    # the device-wide figure also sees other processes' allocations: checked
    # only when this process is alone on the device
    if not _other_processes_on_device(torch):
        assert free1 == free0
    assert out.item() == float(n)
