"""On-device post-processing (dba_tip_profile, dba_size_distribution) against the
CPU restatement of the reference's tools, on fields taken from running simulations."""
import numpy as np
import pytest

import dba_b200
import oracle_lib as ol
from cases import DENDRITE_REF, MODELB_REF, dendrite_cfg, modelb_cfg

pytestmark = pytest.mark.gpu

MB = dict(MODELB_REF, metric_eps=1e-3, chi_zb=3.0, eps_x=1.0, eps_y=1.0, eps_z=1.0, k_0=1e-4, dt=0.0002)


def smooth_z(shape, seed, width=4.0, skew=1.0):
    """x = y = 0.05 and a smooth random z in [0.05, 0.85] (low-pass filtered noise,
    raised to `skew` so that fewer regions cross the threshold)."""
    rng = np.random.default_rng(seed)
    k = [np.fft.fftfreq(n) for n in shape]
    kk = sum(np.meshgrid(*[a * a for a in k], indexing="ij"))
    w = np.real(np.fft.ifftn(np.fft.fftn(rng.standard_normal(shape)) * np.exp(-kk * (2 * np.pi * width) ** 2 / 2)))
    w = (w - w.min()) / (w.max() - w.min())
    z = 0.05 + 0.8 * w ** skew
    return [np.full(shape, 0.05), np.full(shape, 0.05), z]


@pytest.mark.parametrize("prec", [0, 1])
def test_size_distribution_matches_tool_3d(prec):
    s = dba_b200.Simulation(modelb_cfg(MB, 32, 32, 32, 8, precision=prec)).init(smooth_z((32, 32, 32), 5, width=1.5, skew=2.0))
    s.step(20, 1)
    z = s.field("z")
    avg, vol, sizes = s.size_distribution("z")
    oavg, ovol, osizes = ol.size_distribution(z)
    assert avg == oavg and vol == ovol
    assert np.array_equal(sizes, osizes)
    assert len(sizes) > 3


def test_size_distribution_matches_tool_2d_conserved_fp32():
    s = dba_b200.Simulation(modelb_cfg(MB, 128, 128, 1, 16, precision=1, conserved=1)).init(
        [a[None] for a in smooth_z((128, 128), 7, width=3.0)])
    s.step(40, 1)
    z = s.field("z")
    avg, vol, sizes = s.size_distribution("z")
    oavg, ovol, osizes = ol.size_distribution(z)
    assert avg == oavg and vol == ovol
    assert np.array_equal(sizes, osizes)
    assert len(sizes) > 3


@pytest.mark.parametrize("prec", [0, 1])
def test_tip_profile_matches_tool(prec):
    prm = dict(DENDRITE_REF, Delta=1.15, delta=0.2, metric_p=1e-3, metric_T=1e-5)
    cfg = dendrite_cfg(prm, 64, 32, 48, 8, precision=prec, bc=1, ic=1, ic_radius=8.0, ic_width=2.0)
    s = dba_b200.Simulation(cfg).init()
    s.step(700, 1)
    p = s.field("p")
    tip, m = s.tip_profile(dz=40)
    otip, om = ol.tip_profile(p, dz=40)
    assert np.array_equal(tip, otip) and m == om
    assert m > 32                              # the seed (centre x = 32) has grown along +x


def test_union_retry_limit_reports_timeout():
    """The union step of dba_size_distribution retries its compare-and-swap at most
    DBA_OPT_WAIT_LIMIT times; with a limit of 0 every union gives up and dba_sync
    reports DBA_ERR_TIMEOUT instead of a wrong answer passing silently."""
    s = dba_b200.Simulation(modelb_cfg(MB, 32, 32, 32, 8, precision=0)).init(smooth_z((32, 32, 32), 5, width=1.5, skew=2.0))
    s.set_option(dba_b200.OPT_WAIT_LIMIT, 0)
    s.size_distribution("z")
    with pytest.raises(dba_b200.DBAError) as e:
        s.sync()
    assert e.value.code == 6


def _ref_post():
    import os
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(here, "golden"))
    import make_post_golden as mpg
    return mpg, np.load(os.path.join(here, "golden", "ref_post.npz"))


def test_tip_profile_matches_reference_tool():
    """dba_tip_profile on a resident 64^3 field against Tip_Profile.dat of the reference's
    own Extract_Tip on the same field (tests/golden/make_post_golden.py)."""
    mpg, g = _ref_post()
    f = mpg.tip_field()
    s = dba_b200.Simulation(dendrite_cfg(DENDRITE_REF, 64, 64, 64, 8)).init([f, np.zeros_like(f)])
    tip, m = s.tip_profile(40)
    assert np.array_equal(np.stack([np.arange(41), m - tip], axis=1), g["tip_profile"])


@pytest.mark.parametrize("prec", [0, 1])
def test_size_distribution_matches_reference_tool(prec):
    """dba_size_distribution on a resident 256^3 Model B z field against size_dist.txt and
    avg_radius.txt of the reference's own coarsening_analysis on the same field."""
    mpg, g = _ref_post()
    z = mpg.sphere_field(g["spheres"])
    s = dba_b200.Simulation(modelb_cfg(MB, 256, 256, 256, 8, precision=prec)).init(
        [np.full_like(z, 0.03125), np.full_like(z, 0.03125), z])
    avg, vol, sizes = s.size_distribution("z")
    assert np.array_equal(sizes, g["sizes"])
    assert float(f"{np.cbrt(vol * 0.75 / np.pi / len(sizes)):.6g}") == float(g["avg_radius"])
    s.sync()
