"""Continuous batching on the device: requests submitted while others run are
admitted as slots free up, and each result is the same alone and in the mix
(bit for bit: a request's state never depends on the other slots)."""
import copy

import numpy as np
import pytest

from softdft_b200 import native
from softdft_b200.host.descriptor import numerics_from_dict
from tests.helpers import descriptor, small_slit

pytestmark = pytest.mark.gpu


def _cases():
    # parameter points that the CPU oracle solves in 703-2579 iterations; their
    # different iteration counts make requests finish, and slots free up, at
    # different steps.  Trajectories this long depend on rounding (the first
    # least-squares problems are nearly singular), so a device build may end
    # one of them non-finite; the property checked is that each request ends
    # the same alone and in the mix.
    pts = [(7.0, 0.1, 6), (8.0, 0.1, 7), (9.0, 0.2, 8), (4.0, 0.1, 9), (8.5, 0.3, 6)]
    return [small_slit(pH=pH, salt=salt, n_chain=n) for pH, salt, n in pts]


@pytest.mark.parametrize("pipelined", [False, True])
def test_results_alone_equal_results_in_the_mix(pipelined):
    cases = _cases()
    numd = dict(cases[0]["numerical"], tole=1e-8, max_iters=5000)
    num = numerics_from_dict(numd)
    dfts = [descriptor(c) for c in cases]
    alone = []
    for d in dfts:
        s = native.DeviceSystem(d.descriptor)
        try:
            it, err, rc = s.solve(num)
        except native.SdftError as e:
            rc = e.code
            it = s.solver_state()[0].iter
        alone.append((s.get_x(), it, rc))
    assert sum(a[2] == 0 for a in alone) >= 3, [a[1:] for a in alone]
    srv = native.Server(num, max_slots=3)
    srv.set_pipeline(pipelined)
    systems = [native.DeviceSystem(d.descriptor) for d in dfts]
    # staggered submission: two now, the rest while those run
    srv.submit(systems[0], 0)
    srv.submit(systems[1], 1)
    done = {}
    pending = 2
    nxt = 2
    steps = 0
    while len(done) < len(systems):
        active, queued = srv.step(7)
        steps += 1
        for tag, st, it, err, dms in srv.poll():
            done[tag] = (st, it, err)
        if nxt < len(systems) and steps % 2 == 1:
            srv.submit(systems[nxt], nxt)
            nxt += 1
        assert active <= 3
        assert steps < 5000
    for i, s in enumerate(systems):
        st, it, err = done[i]
        assert st == alone[i][2] and it == alone[i][1]
        if st == 0:
            assert err < 1e-8
        assert np.array_equal(s.get_x(), alone[i][0], equal_nan=True)
    srv.close()


def test_byte_budget_limits_admission():
    cases = _cases()[:3]
    num = numerics_from_dict(dict(cases[0]["numerical"], tole=1e-8, max_iters=5000))
    systems = [native.DeviceSystem(descriptor(c).descriptor) for c in cases]
    one = max(s.device_bytes for s in systems)
    srv = native.Server(num, max_slots=8, max_bytes=one)  # room for one request at a time
    for i, s in enumerate(systems):
        srv.submit(s, i)
    done = []
    while len(done) < 3:
        active, queued = srv.step(50)
        assert active <= 1
        done += srv.poll()
    assert sorted(t for t, *_ in done) == [0, 1, 2]
    srv.close()


def test_admission_follows_free_device_memory():
    """Prepared requests take device memory only at admission, and only while
    the free device memory less the server's reserve covers them: with a
    reserve that leaves room for two requests, at most two are active, the
    queue waits for retirements (each finished request is destroyed, and its
    block, kept in the library's cache, serves the next one), and every
    request ends in the state of its solve alone."""
    import torch

    cases = [small_slit(np_=4096, dz=0.005, pH=pH, n_chain=6) for pH in (6.0, 7.0, 8.0, 9.0, 7.5)]
    num = numerics_from_dict(dict(cases[0]["numerical"], tole=1e-8, max_iters=5000))
    dfts = [descriptor(c) for c in cases]
    alone = []
    for d in dfts:
        s = native.DeviceSystem(d.descriptor)
        try:
            it, err, rc = s.solve(num)
        except native.SdftError as e:
            rc = e.code
            it = s.solver_state()[0].iter
        alone.append((s.get_x(), it, rc))
        s.close()
    assert sum(a[2] == 0 for a in alone) >= 3, [a[1:] for a in alone]
    prepared = [native.DeviceSystem(d.descriptor, prepare=True) for d in dfts]
    one = max(s.device_bytes for s in prepared)
    assert one > 16 * 2 ** 20  # large against the 2 MiB allocation granularity
    srv = native.Server(num, max_slots=8)
    native.release_cached_memory()  # the solves above left their blocks in the library's cache
    free0, _ = torch.cuda.mem_get_info()
    srv.set_reserve(int(free0 - 2.5 * one))
    for i, s in enumerate(prepared):
        srv.submit(s, i)
    done = {}
    most = 0
    steps = 0
    while len(done) < len(prepared):
        active, queued = srv.step(40)
        most = max(most, active)
        assert active <= 2
        for tag, st, it, err, dms in srv.poll():
            x = prepared[tag].get_x()
            done[tag] = (st, it, x)
            prepared[tag].close()  # the finished request's memory returns to the pool of free HBM
        steps += 1
        assert steps < 2000
    assert most == 2
    for i in range(len(prepared)):
        st, it, x = done[i]
        assert st == alone[i][2] and it == alone[i][1]
        assert np.array_equal(x, alone[i][0], equal_nan=True)
    srv.close()


def test_destroyed_request_blocks_are_reused_and_released():
    """A destroyed request's device block serves the next request of its size
    without new device memory, a request on a reused block solves to the same
    state bit for bit, and sdft_release_cached_memory hands the blocks back."""
    import torch

    d = descriptor(small_slit(np_=4096, dz=0.005, n_chain=6)).descriptor
    num = numerics_from_dict(dict(small_slit()["numerical"], tole=1e-8, max_iters=200))
    native.release_cached_memory()
    a = native.DeviceSystem(d)
    one = a.device_bytes
    assert one > 16 * 2 ** 20  # large against the 2 MiB allocation granularity
    it_a, _, _ = a.solve(num)
    x_a = a.get_x()
    a.close()  # its block goes to the cache
    free1, _ = torch.cuda.mem_get_info()
    b = native.DeviceSystem(d)  # on that block
    free2, _ = torch.cuda.mem_get_info()
    assert free1 - free2 < one // 2
    it_b, _, _ = b.solve(num)
    assert it_b == it_a and np.array_equal(b.get_x(), x_a)
    b.close()
    released = native.release_cached_memory()
    assert released >= one
    free3, _ = torch.cuda.mem_get_info()
    assert free3 - free2 >= 0.9 * one
    assert native.release_cached_memory() == 0
