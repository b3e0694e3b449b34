"""An allocation that fails is reported and retried, never half-done: the lazily allocated diagnostic
scratch of a case meets a device whose memory is taken (by another user of it, here torch) and the
diagnostic returns ITLBM_E_OOM; once memory is free again the next call allocates and measures."""
import pytest

pytestmark = pytest.mark.gpu


def test_diag_scratch_failure_then_retry(gpu):
    import torch
    op = gpu.make_op(3, 0.5)
    d = gpu.desc(1024, 1024, op, tau=1.0, A_fact=0.225, radius=100.0)
    with gpu.Case(d) as c:
        c.step(2, keep_aux=True)
        c.sync()
        # leave less than the 48 MB the scratch of a 1024^2 drop needs
        hog = None
        for spare_mb in (8, 16, 24, 32):
            free, _ = torch.cuda.mem_get_info()
            try:
                hog = torch.empty(max(0, free - (spare_mb << 20)), dtype=torch.uint8, device="cuda")
                break
            except torch.OutOfMemoryError:
                torch.cuda.empty_cache()
        if hog is None:
            pytest.skip("could not take the device's memory")
        try:
            with pytest.raises(gpu.ItlbmError) as e:
                c.diag_drop(1)
            assert e.value.code == -2  # ITLBM_E_OOM
            with pytest.raises(gpu.ItlbmError):  # still no room: the failed call kept nothing
                c.diag_drop(1)
        finally:
            del hog
            torch.cuda.empty_cache()
        dg = c.diag_drop(1)
        assert dg.ok and dg.raio > 90
