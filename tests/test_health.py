"""Wavefield health check (cgfdm_check_finite, the "checkFinite" option): a
NaN planted in the state through the C ABI (host data, no device fault) is
counted and located, and a run with checkFinite stops at the first scan
after it with CGFDM_E_NONFINITE naming the step; a clean run scans clean."""

import numpy as np
import pytest

import parity_util as pu
from cgfdm import CgfdmError, Session, cases


@pytest.mark.gpu
def test_nonfinite_values_are_found(tmp_path):
    c = pu.small_halfspace(steps=16)
    d = cases.write_case(c, str(tmp_path / "run"))
    with Session(d) as s:
        s.run(4)
        assert s.check_finite() == (0, -1)
        i = s.info
        w = s.wavefield()
        w[3 + 7, 3 + 5, 3 + 9, 4] = np.nan
        w[3 + 8, 3 + 1, 3 + 2, 0] = np.inf
        s.set_wavefield(w)
        n, first = s.check_finite()
        assert n == 2
        assert first == ((7 * i.ny + 5) * i.nx + 9) * 9 + 4
    with Session(d, options='{"checkFinite": 3}') as s:
        s.run(6)                                   # scans after steps 3 and 6: clean
        w = s.wavefield()
        w[3 + 7, 3 + 5, 3 + 9, 4] = np.nan
        s.set_wavefield(w)
        with pytest.raises(CgfdmError) as e:
            s.run(6)
        assert e.value.code == 20005 and "after step 9" in str(e.value)
