"""Host side of the learned-guess workload (no GPU): the many-grain 2D
packing and its colouring."""
import numpy as np

from hpsint_b200 import learned_guess as LG


def test_packing_has_the_workload_shape():
    for seed in (0, 1, 7):
        centers, radii, colours = LG.packing_2d(seed)
        assert len(radii) == 100
        assert radii.min() >= 6.0 and radii.max() <= 12.0
        assert colours.max() + 1 <= 8
        assert np.all(centers - radii[:, None] >= 1.0) and np.all(centers + radii[:, None] <= 511.0)


def test_colouring_separates_touching_grains():
    centers, radii, colours = LG.packing_2d(3)
    d = np.linalg.norm(centers[:, None] - centers[None], axis=-1)
    gap = d - radii[:, None] - radii[None]
    same = colours[:, None] == colours[None]
    np.fill_diagonal(same, False)
    # same order parameter only for grains whose surfaces are >= 4 cells apart
    assert np.all(gap[same] >= 4.0)


def test_lumped_mass_integrates_constants():
    m = LG.lumped_mass_2d(9)
    assert abs(m.sum() - 64.0) < 1e-12
