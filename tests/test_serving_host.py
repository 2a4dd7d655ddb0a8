"""CPU tests of the serving workload's host side: the seeded request stream
(512 requests, Poisson arrivals at 20/s, grids from 64^3 to 384 x 256 x 128
cells, d in {0.02, 0.025, 0.04} um, wavelength 1.50-1.60 um, 3-12 boxes with
sides 0.2-2.0 um, silicon or oxide) and the large grating slab spec."""
import numpy as np

from emopt_b200 import serving as S


def test_stream_matches_the_serving_workload():
    reqs = S.poisson_stream(512, 20.0, seed=3)
    assert len(reqs) == 512 and [r.rid for r in reqs] == list(range(512))
    t = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(t) > 0)
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert abs(gaps.mean() - 1 / 20.0) < 0.1 / 20.0           # 512 draws: well within 10%
    for r in reqs:
        Nz, Ny, Nx = r.shape
        assert 64 <= Nz <= 128 and 64 <= Ny <= 256 and 64 <= Nx <= 384
        assert r.d in (0.02, 0.025, 0.04)
        assert 1.50 <= r.wavelength <= 1.60
        assert 3 <= len(r.boxes) <= 12 and r.w_pml == 15 and r.precision == 32
        for x0, x1, y0, y1, z0, z1, eps in r.boxes:
            for lo, hi in ((x0, x1), (y0, y1), (z0, z1)):
                assert 0.2 - 1e-12 <= hi - lo <= 2.0 + 1e-12
            assert eps in (S.EPS_SI, S.EPS_SIO2)
    # seeded: the same stream every time
    again = S.poisson_stream(512, 20.0, seed=3)
    assert [(r.shape, r.d, r.arrival) for r in again] == [(r.shape, r.d, r.arrival) for r in reqs]


def test_grating_slab_spec():
    g = S.grating_spec()
    assert g.shape == (301, 601, 1201) and g.ncells == 217_262_101
    assert g.w_pml == 25 and g.d == 0.02 and g.wavelength == 1.55
    trenches = g.boxes[2:]
    assert len(trenches) == 40
    assert all(0.1 - 1e-12 <= x1 - x0 <= 0.4 + 1e-12 for x0, x1, *_ in trenches)
    assert g.src_phase_y > 0


def test_request_eps_arrays_voxel_sampling():
    """eps_arrays: SiO2 background, the boxes in order (later ones win),
    each Yee component sampled at its own staggered position (the offsets of
    FDTD.build for eps), on any torch device (here the CPU)."""
    reqs = S.poisson_stream(3, 20.0, seed=5)
    for r in reqs:
        r.shape = (9, 11, 13)                       # small grid, same boxes
        got = [a.numpy() for a in S.eps_arrays(r, "cpu")]
        Nz, Ny, Nx = r.shape
        i, j, k = np.meshgrid(np.arange(Nz), np.arange(Ny), np.arange(Nx), indexing="ij")
        for c, (sx, sy, sz) in enumerate([(0.5, 0.0, -0.5), (0.0, 0.5, -0.5), (0.0, 0.0, 0.0)]):
            x, y, z = (k + sx) * r.d, (j + sy) * r.d, (i + sz) * r.d
            want = np.full(r.shape, S.EPS_SIO2)
            for x0, x1, y0, y1, z0, z1, v in r.boxes:
                want = np.where((x >= x0) & (x <= x1) & (y >= y0) & (y <= y1) & (z >= z0) & (z <= z1), v, want)
            assert np.array_equal(got[c].real, want) and not got[c].imag.any()
