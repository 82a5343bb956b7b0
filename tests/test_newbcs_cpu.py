"""The reference's counter-based noise rand_noseeded
(TSLB_2C-mpi/vars_single_3D_module.f90:150-215): the library's restatement
(tslb_rand_noseeded, also used on the device) equals the statement-by-statement
transcription bit for bit."""
import itertools

import numpy as np

from entropicthreadsafe_b200 import capi
from oracle import newbcs


def test_rand_noseeded_is_bit_exact():
    L = capi.lib()
    vals = (1, 2, 3, 17, 76, 100, 177, 178, 179, 250)
    got, ref = [], []
    for i, j, k, l in itertools.product(vals, vals, (1, 2, 99), (0, 1, 10, 168, 169, 20000)):
        got.append(L.tslb_rand_noseeded(i, j, k, l))
        ref.append(float(newbcs.rand_noseeded(i, j, k, l)))
    got, ref = np.array(got, np.float32), np.array(ref, np.float32)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    # a uniform variate on [0, 1) of 24-bit resolution
    assert got.min() >= 0 and got.max() < 1 and abs(got.mean() - 0.5) < 0.05
    assert np.all(np.round(got * 2 ** 24) == got * 2 ** 24)
