"""hyt_measure_peaks on a B200: every bandwidth measured, positive and
below what the hardware can carry (HBM3e copy < 8 TB/s nominal, host link
< 200 GB/s); the device facts read back."""
from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu


def test_measure_peaks(hyt, gpu):
    p = hyt.measure_peaks(0, 256 << 20)
    assert p["copy_bytes"] == 256 << 20 and p["link_bytes"] == 256 << 20
    assert 500.0 < p["hbm_copy_gbs"] < 9000.0, p
    for k in ("h2d_gbs", "d2h_gbs", "zero_copy_gbs"):
        assert 1.0 < p[k] < 200.0, (k, p)
    assert p["sm_count"] > 0 and p["l2_bytes"] > 0 and p["hbm_bytes"] > (1 << 30)
    with pytest.raises(hyt.HytError) as e:
        hyt.measure_peaks(hyt.device_count())
    assert e.value.code == hyt.capi.HYT_E_INVALID
