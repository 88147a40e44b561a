"""Engine settings (gnd_tune) change speed, never results: every setting renders the
same film sums as the defaults (sum wL and sum w are fixed-point, so bit-equal; the float
sum of wL^2 within 1e-5 relative), for path and volpath, and the autotuner returns valid
settings that keep that property."""
import numpy as np
import pytest

import gianduia_b200 as G
from gianduia_b200 import scenes

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(600)]

DEFAULTS = dict(pool_log2=22, round_iters=8, trav_blocks=8, material_sort=1, stack_smem=32, graphs=1, sample_film=1,
                spec_extend=0, spec_shadow=0, ray_sort=0, leaf_batch=32, trace_leaf_batch=12,
                shadow_leaf_batch=32, trace_blocks=8)
VARIANTS = [dict(material_sort=0), dict(stack_smem=16), dict(trav_blocks=4), dict(pool_log2=16),
            dict(round_iters=2), dict(graphs=0), dict(sample_film=0), dict(spec_extend=1), dict(spec_shadow=1),
            dict(ray_sort=1), dict(ray_sort=3), dict(ray_sort=2, graphs=0, pool_log2=16),
            dict(leaf_batch=16), dict(leaf_batch=1, spec_extend=1), dict(leaf_batch=8, stack_smem=16),
            dict(shadow_leaf_batch=12), dict(shadow_leaf_batch=1, spec_shadow=1),
            dict(trav_blocks=9), dict(trav_blocks=10, leaf_batch=16), dict(trav_blocks=10, spec_extend=1),
            dict(material_sort=0, stack_smem=16, trav_blocks=2, pool_log2=16, round_iters=4, graphs=0)]


@pytest.fixture(scope="module")
def setup(tmp_path_factory):
    d = tmp_path_factory.mktemp("tune")
    ctx = G.GpuContext(0)
    # 64 x 64 x 32 = 131,072 samples: more than a 2^16-slot pool, so refills are exercised
    cb = ctx.upload(G.HostScene.load_xml(scenes.cornell(str(d / "c"), width=64, height=64, spp=32)))
    vol = ctx.upload(G.HostScene.load_xml(scenes.volumetric(str(d / "v"), width=48, height=48, spp=32, max_depth=16)))
    # a 16 x 16 grid of the microfacet spheres: 257 instances, so the top-level tree has
    # several levels and rays enter many bottom-level trees
    grid = ctx.upload(G.HostScene.load_xml(scenes.microfacet(str(d / "g"), width=96, height=96, spp=16, max_depth=8,
                                                              grid=16, seed=3)))
    ctx.grid_sid = grid
    yield ctx, cb, vol
    ctx.close()


def same_film(a, b, label):
    assert np.array_equal(a[..., :4], b[..., :4]), "%s: film sums differ on %d values" % (
        label, int((a[..., :4] != b[..., :4]).sum()))
    np.testing.assert_allclose(a[..., 4:], b[..., 4:], rtol=1e-5, atol=1e-6, err_msg=label)


@pytest.mark.parametrize("which", ["path", "volpath", "instances"])
def test_every_setting_renders_the_same_film(setup, which):
    ctx, cb, vol = setup
    sid = {"path": cb, "volpath": vol, "instances": ctx.grid_sid}[which]
    ctx.set_tune(sid, **DEFAULTS)
    assert ctx.get_tune(sid) == DEFAULTS
    base, st0 = ctx.render(sid, batched=True)
    assert st0["passes"] in (16, 32)
    for v in VARIANTS:
        ctx.set_tune(sid, **DEFAULTS)
        ctx.set_tune(sid, **v)
        f, st = ctx.render(sid, batched=True)
        same_film(f, base, "%s %s" % (which, v))
        # the same paths: the same number of closest-hit and shadow queries
        assert (st["extend_rays"], st["shadow_rays"]) == (st0["extend_rays"], st0["shadow_rays"]), (which, v)
    ctx.set_tune(sid, **DEFAULTS)
    plain, _ = ctx.render(sid, batched=False)
    same_film(plain, base, which + " plain vs batched")


def test_invalid_settings_are_refused(setup):
    ctx, cb, _ = setup
    for bad in (dict(stack_smem=24), dict(round_iters=3), dict(pool_log2=40), dict(trav_blocks=0), dict(sample_film=2)):
        with pytest.raises(G.GndError) as e:
            ctx.set_tune(cb, **bad)
        assert e.value.status == G.GND_ERR_INVALID
    assert ctx.get_tune(cb) == DEFAULTS


def test_autotune(setup):
    ctx, cb, _ = setup
    ctx.set_tune(cb, **DEFAULTS)
    base, _ = ctx.render(cb, batched=True)
    tune, mpaths = ctx.autotune(cb, spp=8, budget_ms=3000)
    assert mpaths > 0
    assert tune == ctx.get_tune(cb)
    assert 16 <= tune["pool_log2"] <= 26 and tune["stack_smem"] in (16, 32) and 1 <= tune["trav_blocks"] <= 8
    f, _ = ctx.render(cb, batched=True)
    same_film(f, base, "after autotune %s" % tune)
    ctx.set_tune(cb, **DEFAULTS)
