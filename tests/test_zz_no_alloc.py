"""sdft_objective_noalloc: G(x) for callers that cannot call cudaMalloc.

Callers whose device memory belongs to another allocator (a framework's pool or
a budget reserved at start-up), or that cannot afford the device
synchronisation a cudaMalloc may cause, get G(x) with every intermediate array
in the library's static device scratch.  This test (collected last, so a
failure here comes after every other test has run) calls the entry point
through the C ABI twice in a row, on two different systems, and checks each
result against the allocating entry point sdft_objective within the G(x)
tolerance of the parity tests (1e-11 relative to max |G|).  x and G(x) live in
device memory the test itself owns (torch tensors).
"""
import copy

import numpy as np
import pytest

from softdft_b200 import native, workloads
from tests.helpers import descriptor, rel, small_slit

pytestmark = pytest.mark.gpu

TOL = 1e-11


def _systems():
    a = small_slit(wall_charge=-0.05)
    b = workloads.grafted_brush(256, 0.05, 10, 0.05, 4.5, 7.0, 0.01)
    return [descriptor(copy.deepcopy(a)), descriptor(copy.deepcopy(b))]


def test_noalloc_matches_allocating_objective_twice():
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    for dft in _systems():
        dev = native.DeviceSystem(dft.descriptor)
        x = dev.get_x()
        g_ref = dev.objective()
        dev.close()
        x_t = torch.from_numpy(x).to("cuda")
        g_t = torch.full_like(x_t, float("nan"))
        torch.cuda.synchronize()
        native.objective_noalloc(dft.descriptor, x_t.data_ptr(), g_t.data_ptr(), 0)
        torch.cuda.synchronize()
        g_new = g_t.cpu().numpy()
        assert np.all(np.isfinite(g_new))
        assert rel(g_new, g_ref) < TOL
        # x is read only
        assert np.array_equal(x_t.cpu().numpy(), x)


def test_noalloc_rejects_oversized_system():
    torch = pytest.importorskip("torch")
    dft = descriptor(workloads.weak_acid_slit(16384, 0.02, 20, 4.5, 7.0, 0.1, 0.3))
    n = dft.descriptor.n_unknowns
    x_t = torch.zeros(n, dtype=torch.float64, device="cuda")
    g_t = torch.zeros(n, dtype=torch.float64, device="cuda")
    with pytest.raises(native.SdftError) as e:
        native.objective_noalloc(dft.descriptor, x_t.data_ptr(), g_t.data_ptr(), 0)
    assert e.value.code == 2 and "scratch" in str(e.value)
