"""Host logic of the job pool (tild_pool_*), no GPU needed: admission checks at submit,
ownership of the box on refusal, and failures reported through the job's status."""
import numpy as np
import pytest

import tild_b200
from tild_b200 import synth


def configured_box(seed=1, **opts):
    o = {"write_files": 0}
    o.update(opts)
    return tild_b200.box_from_spec(synth.small_system(seed=seed, order=3), options=o)


def gpu_visible():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_submit_over_budget_is_refused_and_the_caller_keeps_the_box():
    with tild_b200.Pool(mem_budget_bytes=1 << 20) as pool:   # 1 MiB: smaller than any job
        b = configured_box()
        with pytest.raises(tild_b200.TildError, match="budget") as e:
            pool.submit(b, 10)
        assert e.value.code == 1   # TILD_ERR_ARG
        assert b.N == 160          # the box is still the caller's
        assert pool.stats()["queued"] == 0
        b.close()


def test_submit_argument_errors():
    with tild_b200.Pool(mem_budget_bytes=1 << 30) as pool:
        b = configured_box()
        with pytest.raises(tild_b200.TildError, match="nsteps"):
            pool.submit(b, -1)
        b.close()
        bad = tild_b200.Box(options={"write_files": 0})
        bad.command("Dim 3")
        with pytest.raises(tild_b200.TildError, match="no particles"):
            pool.submit(bad, 5)   # rejected by the host checks of endBox
        bad.close()
        with pytest.raises(tild_b200.TildError, match="no job"):
            pool.status(12345)


@pytest.mark.skipif(gpu_visible(), reason="checks the failure path of a machine without a GPU")
def test_job_fails_loudly_without_a_gpu():
    with tild_b200.Pool(mem_budget_bytes=1 << 30) as pool:
        b = configured_box()
        job = pool.submit(b, 5)
        assert b._h is not None
        with pytest.raises(tild_b200.TildError, match="CUDA"):
            pool.wait(job)
        st = pool.status(job)
        assert st["state"] == "failed" and st["steps_done"] == 0
        assert pool.stats()["failed"] == 1 and pool.stats()["bytes_in_use"] == 0
        pool.release(job)
        b.close()
        with pytest.raises(tild_b200.TildError, match="no job"):
            pool.status(job)


def test_emptied_box_cannot_be_submitted_twice():
    if gpu_visible():
        pytest.skip("the first submit would run")
    with tild_b200.Pool(mem_budget_bytes=1 << 30) as pool:
        b = configured_box()
        pool.submit(b, 1)
        with pytest.raises(tild_b200.TildError, match="already submitted"):
            pool.submit(b, 1)
        b.close()
    assert np.isfinite(1.0)


def test_cancel_and_budget_argument_errors():
    with tild_b200.Pool(mem_budget_bytes=1 << 30) as pool:
        with pytest.raises(tild_b200.TildError, match="no job"):
            pool.cancel(777)
        with pytest.raises(tild_b200.TildError, match="budget"):
            pool.set_budget(-1)
        pool.set_budget(1 << 20)
        assert pool.stats()["budget"] == 1 << 20 and pool.stats()["cancelled"] == 0
        b = configured_box()
        with pytest.raises(tild_b200.TildError, match="budget"):   # checked against the new budget
            pool.submit(b, 5)
        b.close()


@pytest.mark.skipif(gpu_visible(), reason="checks the failure path of a machine without a GPU")
def test_cancel_after_failure_is_refused():
    with tild_b200.Pool(mem_budget_bytes=1 << 30) as pool:
        b = configured_box()
        job = pool.submit(b, 5)
        with pytest.raises(tild_b200.TildError):
            pool.wait(job)
        with pytest.raises(tild_b200.TildError, match="already finished") as e:
            pool.cancel(job)
        assert e.value.code == 5   # TILD_ERR_STATE
        b.close()
