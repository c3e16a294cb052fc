"""Host-side checks of the FP32-mixed ensemble API (no GPU): which configurations
the FP32 form accepts."""
import pytest

from penguin_b200 import params as P
from penguin_b200._lib import PG_ERR_CONFIG, PGError
from penguin_b200.ensemble import check_params


def test_planet_disks_are_accepted():
    check_params([P.planet_disk(128, 384), P.planet_disk(256, 768, q=1e-5, alpha=1e-2, h=0.08)])


def test_seeded_ensemble_has_the_configured_ranges():
    ps = P.disk_ensemble()
    assert len(ps) == 48
    assert all(p.xres % 32 == 0 and 128 <= p.xres <= 512 and p.yres == 3 * p.xres for p in ps)
    assert all(1e-5 <= p.planet_mass <= 3e-3 and 1e-4 <= p.ss_alpha <= 1e-2 and 0.03 <= p.sc_h <= 0.08 for p in ps)
    check_params(ps)


@pytest.mark.parametrize("bad, why", [
    (P.sod_tube(1024), "ndim 2"),
    (P.planet_disk(128, 384).replace(EOS_flag=2), "isothermal"),
    (P.planet_disk(128, 384).replace(cool_flag=1), "no cooling"),
    (P.planet_disk(128, 384).replace(twobd_flag=1), "fixed star"),
    (P.planet_disk(128, 384).replace(bound_lft=1), "bound 0"),
    (P.planet_disk(128, 384).replace(OrbAdv_flag=0), "orbital advection"),
    (P.planet_disk(32, 96), "at least 64"),
])
def test_other_configurations_are_rejected(bad, why):
    with pytest.raises(PGError) as ei:
        check_params([P.planet_disk(128, 384), bad])
    assert ei.value.status == PG_ERR_CONFIG
    assert why in str(ei.value) and "disk 1" in str(ei.value)
