"""Failure handling on the GPU, with no GPU fault: errors are injected on the
host (CMH_FAULT) or made by tightening the bounds of the device loops that
retry or wait (cmh_plan_set_limits), and every case checks the status code
and then that the same plan (or a new call) gives the oracle's catalog once
the fault is gone.

* alloc    -> CMH_ERR_OUT_OF_MEMORY (4), no device memory left allocated
* overflow -> CMH_ERR_CAPACITY (6) after the plan's repeated attempts, as a
              rank whose receive buffer overflows stops (read_data.c:551-556)
* a union that may not be attempted -> CMH_ERR_DEVICE_TIMEOUT (7)
* lookback: one cell-sort tile publishes nothing and the next tile's wait,
  bounded to a few polls, runs out -> CMH_ERR_DEVICE_TIMEOUT (7); every
  later kernel of that run returns at once
* per-box status of a batch: a bad box is rejected on its own and the others
  run."""
import numpy as np
import pytest

import cm_halofinder_b200 as cmh
from cm_halofinder_b200 import FofConfig, Plan, fof, synth
from oracle import cpu
from tests.helpers import assert_same_catalog

pytestmark = pytest.mark.gpu

OOM, CAPACITY, TIMEOUT, INVALID = 4, 6, 7, 1


@pytest.fixture(scope="module")
def box():
    w = synth.config2(seed=301, scale=60000 / 256 ** 3)
    return w, cpu.run(w)


@pytest.fixture
def fault(monkeypatch):
    def set_fault(value):
        if value is None:
            monkeypatch.delenv("CMH_FAULT", raising=False)
        else:
            monkeypatch.setenv("CMH_FAULT", value)
    yield set_fault
    monkeypatch.delenv("CMH_FAULT", raising=False)


def device(w):
    import torch
    dev = torch.device("cuda", 0)
    return torch.from_numpy(w.pos).to(dev), torch.from_numpy(w.vel).to(dev)


def test_alloc_fault_then_recovery(box, fault):
    import torch
    w, ref = box
    cfg = FofConfig.from_workload(w)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    fault("alloc")
    with pytest.raises(cmh.CmhError) as e:
        fof(w.pos, w.vel, cfg, members=True)
    assert e.value.status == OOM
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] >= free0 - (64 << 20)  # nothing kept
    fault(None)
    assert_same_catalog(fof(w.pos, w.vel, cfg, members=True), ref)


def test_overflow_fault_then_recovery(box, fault):
    w, ref = box
    pos, vel = device(w)
    plan = Plan(FofConfig.from_workload(w))
    try:
        fault("overflow")
        with pytest.raises(cmh.CmhError) as e:
            plan.run(pos, vel, members=True)
        assert e.value.status == CAPACITY
        fault(None)
        for _ in range(2):   # eager, then the captured graph
            assert_same_catalog(plan.run(pos, vel, members=True), ref)
    finally:
        plan.close()


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_union_bound_runs_out_then_recovery(box, precision):
    w, ref = box
    pos, vel = device(w)
    plan = Plan(FofConfig.from_workload(w, precision=precision))
    try:
        assert_same_catalog(plan.run(pos, vel, members=True), ref)
        plan.set_limits(union_attempts=0)
        with pytest.raises(cmh.CmhError) as e:
            plan.run(pos, vel, members=True)
        assert e.value.status == TIMEOUT and "union" in str(e.value)
        plan.set_limits()
        for _ in range(2):
            assert_same_catalog(plan.run(pos, vel, members=True), ref)
    finally:
        plan.close()


def test_lookback_wait_runs_out_then_recovery(box, fault):
    """The cell sort's second tile publishes nothing; the third tile polls
    it at most 64 times, gives up, and the run reports the timeout instead
    of using an order that is not one."""
    w, ref = box
    pos, vel = device(w)
    plan = Plan(FofConfig.from_workload(w))
    try:
        assert_same_catalog(plan.run(pos, vel, members=True), ref)  # graph captured
        plan.set_limits(lookback_polls=64)
        fault("lookback")
        for _ in range(2):
            with pytest.raises(cmh.CmhError) as e:
                plan.run(pos, vel, members=True)
            assert e.value.status == TIMEOUT and "look-back" in str(e.value)
        fault(None)
        plan.set_limits()
        for _ in range(2):
            assert_same_catalog(plan.run(pos, vel, members=True), ref)
    finally:
        plan.close()


def test_batch_status_rejects_one_box_and_runs_the_others():
    boxes = [synth.config2(seed=310 + i, scale=20000 / 256 ** 3) for i in range(3)]
    cfgs = [FofConfig.from_workload(b) for b in boxes]
    cfgs[1].linklength = 0.0          # invalid: rejected on its own
    pos, vel = zip(*[device(b) for b in boxes])
    plan = Plan(cfgs[0])
    try:
        for _ in range(2):
            cats, status = plan.run_batch(cfgs, list(pos), list(vel), with_status=True)
            assert status == [0, INVALID, 0] and cats[1] is None
            for b in (0, 2):
                ref = cpu.run(boxes[b])
                assert cats[b].nhalos == ref["halo_head"].shape[0] > 0
                np.testing.assert_array_equal(cats[b].head, ref["halo_head"])
        # the strict entry point fails the whole call on the same input
        with pytest.raises(cmh.CmhError) as e:
            plan.run_batch(cfgs, list(pos), list(vel))
        assert e.value.status == INVALID
    finally:
        plan.close()
