"""FP64 diagnostics queued without a host wait (tslb_reduce_async /
tslb_reduce_collect) equal the blocking ones step by step, bit for bit (the
reduction sums in a fixed order), and the queue reports when it is full."""
import pytest

from entropicthreadsafe_b200 import capi, workloads
from entropicthreadsafe_b200.solver import Lattice, TslbError

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [capi.PREC_FP32, capi.PREC_BF16])
def test_queued_diagnostics_equal_blocking_ones(prec):
    p, f = workloads.droplet(n=24, radius=6.0)
    p.precision = prec
    with Lattice(p, 24, 24, 24) as a, Lattice(p, 24, 24, 24) as b:
        a.upload_moments(f)
        b.upload_moments(f)
        blocking = []
        for _ in range(7):
            a.step(1)
            blocking.append(a.reduce())
        for _ in range(7):
            b.step(1)
            b.reduce_async()
        queued = b.reduce_collect()
        assert queued == blocking
        assert b.reduce_collect() == []


def test_full_queue_is_an_error_not_an_overwrite():
    p, f = workloads.droplet(n=16, radius=4.0)
    with Lattice(p, 16, 16, 16) as lat:
        lat.upload_moments(f)
        for _ in range(capi.REDUCE_QUEUE):
            lat.reduce_async()
        with pytest.raises(TslbError) as e:
            lat.reduce_async()
        assert e.value.code == capi.ERR_STATE
        assert len(lat.reduce_collect()) == capi.REDUCE_QUEUE
