"""The ELFS merge/split variant (main/merge_split_ops.h) on the GPU against
the oracle, whose ELFS restatement is pinned bitwise to the reference's own
code (tests/golden/ms_elfs_bench1000.json).  Standalone calls with the ELFS
defaults (a binding max_ops of 50), without a cap and with the divergence
trigger, and the gpu_offload cadence inside the step loop.  Bitwise."""
import numpy as np
import pytest

from amsc_b200 import scenarios
from amsc_b200.dampm import Solver
from oracle.oracle import Oracle

FIELDS = ("x", "y", "vpx", "vpy", "hp", "F_11", "F_12", "F_21", "F_22", "Mp", "Vp", "H",
          "Ap", "mom_px", "mom_py", "Fb_x", "Fb_y", "label", "level",
          "vpx_dx", "vpx_dy", "vpy_dx", "vpy_dy", "xp", "yp")

# ms_config values of main/merge_split_ops.h:17-30 as DATA keys
CONFIGS = {
    "defaults": dict(ms_alpha=2.0, ms_beta=3.0, ms_hp_min=0.05, ms_max_dv=0.01,
                     ms_stretch_thresh=1e7, ms_max_ops=50.0),
    "uncapped": dict(ms_alpha=2.0, ms_beta=3.0, ms_hp_min=0.05, ms_max_dv=0.01,
                     ms_stretch_thresh=1e7, ms_max_ops=1e9),
    "stretch": dict(ms_alpha=1.0, ms_beta=2.0, ms_hp_min=0.05, ms_max_dv=0.05,
                    ms_stretch_thresh=0.5, ms_max_ops=1e9),
}


def elfs_data(config, d=None):
    d = d or scenarios.bench_slab(1000, nsteps=100)
    d.scalars.update(CONFIGS[config])
    d.scalars.update({"ms_variant": 1, "ms_min_level": -2, "ms_max_level": 2,
                      "MERGE_SPLIT_ON": 1})
    return d


def compare(s, o, fields=FIELDS):
    assert s.num_particles == o.np
    for k in fields:
        np.testing.assert_array_equal(s.download(k), o.get(k), err_msg=k)


@pytest.mark.gpu
@pytest.mark.parametrize("config", list(CONFIGS))
def test_elfs_standalone(cuda_lib, config):
    d = elfs_data(config)
    o = Oracle(d, threads=4)
    o.run(12)
    with Solver(d, record=True, capacity=8 * d.np) as s:
        s.step(12)
        cg = s.merge_split(1e-3)
        co = o.merge_split(1e-3)
        assert cg == co, (cg, co)
        assert co[0] > 0 and co[1] > 0 and co[3] != co[2]
        if config == "defaults":
            assert co[0] == 50  # the split cap binds
        compare(s, o)
        # the steps after a merge/split read the emitted Ap/mom/Fb
        s.step(3)
        o.run(3)
        compare(s, o, FIELDS[:17])


@pytest.mark.gpu
def test_elfs_cadence_mudflow(cuda_lib):
    """ELFS at the cadence (every 10 steps) on the 256^2 mudflow: a free
    surface inside a larger grid, so the exterior fill and the distance
    search run over many cells and levels.  Three calls in 35 steps."""
    d = elfs_data("defaults", scenarios.mudflow(N=256))
    o = Oracle(d, threads=4, merge_split=True)
    o.run(35)
    with Solver(d, merge_split=True, capacity=4 * d.np) as s:
        s.step(35)
        st = s.status()
        assert st["it"] == o.it and st["np"] == o.np
        assert o.np != d.np
        compare(s, o, FIELDS[:19])


@pytest.mark.gpu
def test_unknown_variant_is_refused(cuda_lib):
    d = scenarios.bench_slab(1000, nsteps=10)
    with Solver(d) as s:
        assert cuda_lib.dampm_set_ms_variant(s.h, 7, 1e7) == -1     # DAMPM_ERR_ARG
        assert cuda_lib.dampm_set_ms_variant(s.h, 1, 1e7) == 0      # DAMPM_MS_ELFS
        assert cuda_lib.dampm_set_ms_variant(s.h, 0, 1e7) == 0      # back to the default
