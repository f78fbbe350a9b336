"""GPU test of the tile-shape autotuner (shtools_b200.autotune): it times the
candidate shapes of a plan, applies the fastest, and the tuned plan still
reproduces the oracle; real and complex plans."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_autotune_real_and_complex_plans(cuda, oracle, tmp_path, monkeypatch):
    from shtools_b200 import autotune, transforms as T
    monkeypatch.setenv("SHTC_TUNE_CACHE", str(tmp_path / "tune.json"))
    L = 95
    for cplx in (False, True):
        p = T.Plan(T.GRID_DH, L, L, 1, 1, 2, 0, cplx=cplx)
        r = autotune.tune_plan(p, reps=1, use_cache=True)
        assert r["synth_T"] in (1, 2, 4, 8) and r["anal_T"] in (1, 2, 4, 8)
        assert r["anal_W"] in (1, 2, 4, 8)
        assert any(k.startswith("anal_T") for k in r["times_ms"])
        # a second call is answered from the cache
        assert autotune.tune_plan(p, reps=1, use_cache=True)["synth_T"] == r["synth_T"]
        if cplx:
            c = oracle.power_law_cilm_complex(L, 70)
            g = p.synthesis_c(torch.from_numpy(c[None]).cuda())[0].cpu().numpy()
            ref = oracle.makegrid_dhc(c, sampling=2)
        else:
            c = oracle.power_law_cilm(L, 70)
            g = p.synthesis(torch.from_numpy(c[None]).cuda())[0].cpu().numpy()
            ref = oracle.makegrid_dh(c, sampling=2)
        assert np.abs(g - ref).max() / np.abs(ref).max() < 1e-12
