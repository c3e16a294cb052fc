"""File names of snapshots (create_label, src/output/output.cu:14-92; frame_num,
src/util/util.cu:25-36) and the checkpoint layout round trip on the host."""
import numpy as np

from penguin_b200 import params as P
from penguin_b200 import snapshot as S


def test_labels_follow_create_label():
    # 1000 h = 50.000000000000007 -> 50; q / JupiterMass = 1.048 -> 1 J; 10 log10(alpha) = -30
    assert S.label(P.planet_disk(1024, 3072)) == "1024x3072_h50_1p1J_e0_a-30_OA_PPM4"
    # q below a Jupiter mass in Earth masses; Stokes number label
    p = P.dust_disk(768, 2048, stokes=0.01)
    assert S.label(p) == f"768x2048_h50_1p{int(3.0e-4 / 3.0e-6)}E_e0_a-40_OA_St-20_PPM4"
    assert S.file_name(P.planet_disk(64, 192), 7) == "binary_64x192_h50_1p1J_e0_a-30_OA_PPM4_00007"
    assert S.file_name(P.planet_disk(64, 192), 12, average=True).endswith("_ave_00012")


def test_checkpoint_layout_round_trip(tmp_path):
    p = P.planet_disk(8, 12)
    xa = np.linspace(0.4, 2.5, 9)
    ya = np.linspace(0.0, 6.28, 13)
    rng = np.random.default_rng(0)
    f = {k: rng.uniform(size=(12, 8)) for k in ("r", "p", "u", "v")}
    path = tmp_path / "snap"
    S.write_snapshot(str(path), 1.25, xa, ya, f, 2)
    g = S.read_snapshot(str(path), 8, 12, 2)
    assert g["t"] == 1.25 and np.array_equal(g["xa"], xa) and np.array_equal(g["ya"], ya)
    for k in f:
        assert np.array_equal(g[k], f[k])
    assert path.stat().st_size == 8 * (1 + 9 + 13 + 4 * 96)
    del p
