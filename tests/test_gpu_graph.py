"""One captured CUDA graph for a mixed batch (fit_star cutouts + star groups) and
its launch-shape tuner, through the C-ABI.

The graph's results must equal those of the direct batch entry points on the
same inputs: bit-identical for the fit_star half (one warp per cutout, no
cross-cutout arithmetic), and for the group half identical to 1e-9 relative
(the tuner may pick a different block size, which changes only the order of
the in-block reductions).  Replays after refilling the bound inputs fit the new
inputs.  A second construction with the same tuning cache times nothing.
"""
import numpy as np
import pytest

import crowdphot_b200 as cpb
from crowdphot_b200.photometry import _lm_outputs, group_outputs
from crowdphot_b200.simulate import lm_cutouts, lm_groups, moffat_epsf

pytestmark = pytest.mark.gpu


def to_dev(d, keys):
    import torch
    return {k: torch.from_numpy(np.ascontiguousarray(d[k])).cuda() for k in keys}


def lm_half(psf, n, seed):
    import torch
    d = lm_cutouts(n, seed=seed, psf=psf)
    t = to_dev(dict(offsets=d["offsets"], ny=d["ny"], nx=d["nx"], y1=d["y1"], x1=d["x1"], pix=d["pix"],
                    inv_var=d["inv_var"], init=d["init"]), ["offsets", "ny", "nx", "y1", "x1", "pix", "inv_var", "init"])
    t["out"] = {k: torch.from_numpy(v).cuda() for k, v in _lm_outputs(n, 4, 3).items()}
    return d, t


def group_half(n, seed):
    import torch
    d = lm_groups(n, seed=seed)
    t = to_dev(dict(offsets=d["offsets"], ny=d["ny"], nx=d["nx"], pix=d["pix"], inv_var=d["inv_var"],
                    star_offsets=d["star_offsets"], y=d["y"], x=d["x"], flux=d["flux"]),
               ["offsets", "ny", "nx", "pix", "inv_var", "star_offsets", "y", "x", "flux"])
    t["out"] = {k: torch.from_numpy(v).cuda()
                for k, v in group_outputs(int(d["star_offsets"][-1]), n).items()}
    return d, t


GKW = dict(fixed={"bkg": 0.0}, model_rad=12)


def check_against_direct(psf, dl, tl, dg, tg):
    ref_lm = cpb.fit_star_packed(psf, dl["pix"], dl["offsets"], dl["ny"], dl["nx"], dl["y1"], dl["x1"], dl["init"],
                                 inv_var=dl["inv_var"], fixed={"bkg": 0.0})
    for k in ("params", "iterations", "converged", "status", "cost"):
        assert np.array_equal(tl["out"][k].cpu().numpy(), ref_lm[k]), k
    ref_g = cpb.fit_groups_packed(psf, dg["pix"], dg["offsets"], dg["ny"], dg["nx"], dg["star_offsets"], dg["y"],
                                  dg["x"], dg["flux"], 5, inv_var=dg["inv_var"], **GKW)
    G = len(dg["ny"])
    for k in ("n_active", "n_union", "status", "n_failed"):
        assert np.array_equal(tg["out"][k].cpu().numpy()[:G], ref_g[k]), k
    assert (tg["out"]["n_passes"].cpu().numpy()[:G] == ref_g["n_passes"]).mean() > 0.98
    ns = int(dg["star_offsets"][-1])
    same = (tg["out"]["n_iter"].cpu().numpy()[:ns] == ref_g["n_iter"])
    assert same.mean() > 0.99
    for k in ("y", "x", "flux", "spread_model"):
        a = tg["out"][k].cpu().numpy()[:ns][same]
        b = ref_g[k][same]
        np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-9, equal_nan=True)


def test_graph_matches_direct_entries_and_replays_new_inputs(tmp_path):
    psf = moffat_epsf()
    dl, tl = lm_half(psf, 3000, 41)
    dg, tg = group_half(300, 42)
    cache = tmp_path / "tune.txt"
    g = cpb.BatchGraph(psf, lm=tl, lm_fixed={"bkg": 0.0}, groups=tg, fit_rad=5, group_kw=GKW, autotune=1,
                       cache_path=cache)
    info = g.tune_info()
    assert info["n_timed"] >= 3 and info["from_cache"] == 0
    assert info["grp_threads"] in (64, 128, 256) and info["lm_blocks_per_sm"] in (1, 2)
    t = g.launch()
    assert t > 0
    check_against_direct(psf, dl, tl, dg, tg)
    # refill the bound inputs in place (moved initial guesses) and replay
    dl2, dg2 = dict(dl), dict(dg)
    dl2["init"] = dl["init"].copy()
    dl2["init"][:, :2] += 0.07
    for k in ("y", "x"):
        dg2[k] = dg[k] + 0.05
    tl["init"].copy_(tl["init"].new_tensor(dl2["init"]))
    for k in ("y", "x"):
        tg[k].copy_(tg[k].new_tensor(dg2[k]))
    g.launch()
    check_against_direct(psf, dl2, tl, dg2, tg)
    g.close()
    # same signature again: the cached shapes, nothing timed
    g2 = cpb.BatchGraph(psf, lm=tl, lm_fixed={"bkg": 0.0}, groups=tg, fit_rad=5, group_kw=GKW, autotune=1,
                        cache_path=cache)
    info2 = g2.tune_info()
    assert info2["from_cache"] == 1 and info2["n_timed"] == 0
    assert (info2["grp_threads"], info2["grp_blocks_per_sm"]) == (info["grp_threads"], info["grp_blocks_per_sm"])
    g2.close()


def test_graph_single_halves_and_refusal():
    import torch
    psf = moffat_epsf()
    dl, tl = lm_half(psf, 500, 7)
    g = cpb.BatchGraph(psf, lm=tl, lm_fixed={"bkg": 0.0}, autotune=0)
    g.launch()
    ref = cpb.fit_star_packed(psf, dl["pix"], dl["offsets"], dl["ny"], dl["nx"], dl["y1"], dl["x1"], dl["init"],
                              inv_var=dl["inv_var"], fixed={"bkg": 0.0})
    assert np.array_equal(tl["out"]["params"].cpu().numpy(), ref["params"])
    g.close()
    dg, tg = group_half(40, 8)
    g = cpb.BatchGraph(psf, groups=tg, fit_rad=5, group_kw=GKW, autotune=0)
    g.launch()
    g.launch()
    ref = cpb.fit_groups_packed(psf, dg["pix"], dg["offsets"], dg["ny"], dg["nx"], dg["star_offsets"], dg["y"],
                                dg["x"], dg["flux"], 5, inv_var=dg["inv_var"], **GKW)
    ns = int(dg["star_offsets"][-1])
    assert np.array_equal(tg["out"]["flux"].cpu().numpy()[:ns], ref["flux"])
    g.close()
    # a group of 70 stars cannot run in one block: refused for capture
    big = dict(offsets=torch.zeros(1, dtype=torch.int64), ny=torch.full((1,), 120, dtype=torch.int32),
               nx=torch.full((1,), 120, dtype=torch.int32), pix=torch.zeros(14400, dtype=torch.float32),
               star_offsets=torch.tensor([0, 70], dtype=torch.int64),
               y=torch.linspace(5, 115, 70, dtype=torch.float64), x=torch.linspace(5, 115, 70, dtype=torch.float64),
               flux=torch.full((70,), 100.0, dtype=torch.float64))
    big = {k: v.cuda() for k, v in big.items()}
    big["out"] = {k: torch.from_numpy(v).cuda() for k, v in group_outputs(70, 1).items()}
    with pytest.raises(cpb.ArgumentError, match="too large for one thread block"):
        cpb.BatchGraph(psf, groups=big, fit_rad=5, group_kw=GKW, autotune=0)
