"""Short-scan reconstruction with Parker weights (SliceReconstructor(parker=True)): the
GPU path against the oracle fed the oracle's weights (rel-L2 <= 1e-4, the bar of every
cone-beam slice), a short scan reconstructing the same object as the full turn while the
unweighted short scan does not, and raw counts through the correction + weights + filter."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import phantom as oph
from oracle.parker import parker
from oracle.recon import OracleReconstructor
from tomography_local_demo_b200 import SliceReconstructor, circular_cone_vectors

pytestmark = pytest.mark.gpu

PH = oph.Phantom(scale=40.0)
R, C = 48, 64


def _geoms():
    short = circular_cone_vectors(220, 300.0, 600.0, R, C, 2.0, angular_range=np.pi + 0.40)
    full = circular_cone_vectors(440, 300.0, 600.0, R, C, 2.0)
    return short, full


PLANES = [((0.0, 0.0, 0.0), (0.0, 0.0, 1.0)), ((2.0, -1.0, 3.0), (0.3, 0.5, 1.0)), ((0.0, 0.0, 0.0), (1.0, 0.0, 0.0))]


def test_parker_matches_oracle_and_the_full_turn(cuda):
    short, full = _geoms()
    ps = oph.project_cone(PH, short.vectors, R, C)
    pf = oph.project_cone(PH, full.vectors, R, C)
    rec = SliceReconstructor(ps, short, parker=True, verbose=False)
    plain = SliceReconstructor(ps, short, verbose=False)
    ref_full = SliceReconstructor(pf, full, verbose=False)
    w = parker(short.vectors, C)
    oracle = OracleReconstructor((ps * w[None, :, :]).astype(np.float32), short)
    for o, nrm in PLANES:
        got, _ = rec.reconstruct_plane(o, nrm, n=64)
        want, _ = oracle.reconstruct_plane(o, nrm, n=64)
        assert rel_l2(got, want) < 1e-4
        f, _ = ref_full.reconstruct_plane(o, nrm, n=64)
        u, _ = plain.reconstruct_plane(o, nrm, n=64)
        e_parker, e_plain = rel_l2(got, f), rel_l2(u, f)
        assert e_parker < 0.15 and e_plain > 1.5 * e_parker, (e_parker, e_plain)


def test_parker_raw_counts_and_input_untouched(cuda):
    short, _ = _geoms()
    p = oph.project_cone(PH, short.vectors, R, C) * 0.02          # line integrals
    rng = np.random.default_rng(4)
    flat = np.full((2, R, C), 40000, np.uint16)
    dark = np.full((2, R, C), 100, np.uint16)
    counts = (100.0 + 39900.0 * np.exp(-p.transpose(1, 0, 2)))
    raw = np.clip(np.round(counts + rng.normal(0, 5, counts.shape)), 0, 65535).astype(np.uint16)
    a = SliceReconstructor(None, short, parker=True, verbose=False)
    a.set_flat_dark(flat, dark)
    a.add_raw_projections(np.arange(short.n_angles), torch.from_numpy(raw.view(np.int16)).cuda())
    # the fused ingest's correction without the filter: gain = 1 / max(F - D, 1), no row flip
    gain = (1.0 / np.maximum(flat[0].astype(np.float32) - dark[0].astype(np.float32), 1.0)).astype(np.float32)
    lines = -np.log(np.maximum((raw.astype(np.float32) - dark[0].astype(np.float32)) * gain, np.float32(1e-3)))
    lines = lines.transpose(1, 0, 2)                                  # [R, k, C]
    b = SliceReconstructor(None, short, parker=True, verbose=False)
    blk = torch.from_numpy(np.ascontiguousarray(lines)).cuda()
    keep = blk.clone()
    b.add_projections(np.arange(short.n_angles), blk)
    assert torch.equal(blk, keep)                                    # the caller's block is not weighted
    # the same counts in bit-reversed arrival order, in three calls: plateau views go through
    # the fused ingest, the ramped ones through correction + weights + filter, in any mix
    from tomography_local_demo_b200.stream import arrival_order
    c = SliceReconstructor(None, short, parker=True, verbose=False, filter="tc")
    c.set_flat_dark(flat, dark)
    order = arrival_order(short.n_angles, "interleaved")
    for part in np.array_split(order, 3):
        c.add_raw_projections(part, torch.from_numpy(raw[part].view(np.int16)).cuda())
    assert c.n == short.n_angles
    assert 0 < c._parker_flat.sum() < short.n_angles
    for o, nrm in PLANES:
        want = b.reconstruct_plane(o, nrm, n=48)[0]
        assert rel_l2(a.reconstruct_plane(o, nrm, n=48)[0], want) < 1e-5
        assert rel_l2(c.reconstruct_plane(o, nrm, n=48)[0], want) < 5e-5


def test_parker_option_errors(cuda):
    from tomography_local_demo_b200 import ParallelGeometry
    with pytest.raises(ValueError):
        SliceReconstructor(None, ParallelGeometry(np.arange(10) * 0.3, 8, 8), parker=True, verbose=False)
    with pytest.raises(ValueError, match="full turn"):
        SliceReconstructor(None, circular_cone_vectors(50, 300.0, 600.0, 8, 16, 3.0), parker=True, verbose=False)
