"""Launch configuration and autotuner: the chosen grouping of edge slots and elements into blocks
must not change any result (bitwise).  The edge-pass forms (a thread per slot and point, at two
register budgets; a lane pair per slot; a lane per point over records staged in shared memory)
evaluate the same expressions in the same order; the compiler's instruction selection may still
differ between the kernels (measured: up to 1 ulp in a residual), so the lane-pair and staged forms
agree bitwise in FP32 and to 1e-14 relative in FP64, and the point form compiled for 64 registers
agrees with it to 1e-14 in FP64 and to FP32 round-off (1e-5 after 6 steps) in FP32."""
import numpy as np
import pytest

from dgm_in_rust_b200 import Batch, DgmError, build_solver
from dgm_in_rust_b200.workloads import Instance, instance_mesh

CONFIGS = [(256, 0, 256), (64, 0, 64), (128, 7, 128), (96, 1, 32), (32, 3, 160)]


def _advance(mesh, init, order, precision, steps, config=None, tune=False, form=None):
    s = build_solver(mesh, order, 1.4, 0.1, 1.0e30, steps, precision=precision)
    try:
        sd, td = s.spatial_disc, s.temporal_disc
        td.set_initial_on_device(init)
        if form is not None:
            sd.set_edge_form(form)
            assert sd.launch_config["edge_form"] == form
        if config is not None:
            sd.set_launch_config(*config)
            assert tuple(sd.launch_config.values())[:3] == config
        if tune:
            chosen = sd.autotune(repeats=3)
            assert chosen["edge_us"] > 0 and chosen["element_us"] > 0
            assert chosen["element_threads"] in (64, 128, 256)
        td.advance(steps)
        td.synchronize()
        U = sd.new_state()
        td.download(U)
        return U, td.current_time
    finally:
        s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_launch_config_does_not_change_results(built, order, precision):
    mesh, init = instance_mesh(Instance(40, 20, 0.8, 1.25, order))
    U0, t0 = _advance(mesh, init, order, precision, 6)
    for cfg in CONFIGS[1:]:
        for form in ("point", "pair", "staged", "point_r64"):
            U, t = _advance(mesh, init, order, precision, 6, config=cfg, form=form)
            if form == "point_r64" and precision == "fp32":  # FP32 round-off, 6 steps
                assert abs(t - t0) <= 1e-6 * t0 and np.abs(U - U0).max() <= 1e-5 * np.abs(U0).max(), (cfg, form)
            elif form != "point" and precision == "fp64":
                assert abs(t - t0) <= 1e-14 * t0 and np.abs(U - U0).max() <= 1e-14 * np.abs(U0).max(), (cfg, form)
            else:
                assert t == t0 and np.array_equal(U, U0), (cfg, form)
    U, t = _advance(mesh, init, order, precision, 6, tune=True)
    assert abs(t - t0) <= 1e-14 * t0 and np.abs(U - U0).max() <= 1e-14 * np.abs(U0).max()


@pytest.mark.gpu
def test_launch_config_rejects_bad_values(built):
    mesh, init = instance_mesh(Instance(16, 8, 0.5, 2.0, 2))
    s = build_solver(mesh, 2, 1.4, 0.1, 1.0, 5)
    try:
        for bad in [(0, 0, 256), (48, 0, 256), (512, 0, 256), (256, -1, 256), (256, 0, 288)]:
            with pytest.raises(DgmError):
                s.spatial_disc.set_launch_config(*bad)
        assert s.spatial_disc.launch_config == {"edge_threads": 256, "edge_blocks": 0, "element_threads": 256,
                                                "limiter_detector": "compact", "limiter_schedule": "barrier",
                                                "edge_form": "point", "limiter_grid": "full"}
        sd = s.spatial_disc
        assert sd._lib.dgm_set_edge_variant(sd.ctx, 4) == 7  # DGM_BAD_ARG
        with pytest.raises(ValueError):
            sd.set_edge_form("tiles")
        assert sd._lib.dgm_set_limiter_variant(sd.ctx, 2) == 7  # DGM_BAD_ARG
        assert sd._lib.dgm_set_limiter_schedule(sd.ctx, 2) == 7
        assert sd._lib.dgm_set_limiter_grid(sd.ctx, 2) == 7
    finally:
        s.close()


@pytest.mark.gpu
def test_batch_autotune_keeps_results(built):
    insts = [Instance(24, 12, 0.6, 1.0, 2), Instance(32, 16, 0.8, -2.0, 2)]
    built_ = [instance_mesh(i) for i in insts]

    def run(tune):
        b = Batch([m for m, _ in built_], 2, 1.4, [0.1] * 2, [1.0e30] * 2, [5] * 2, precision="fp32")
        try:
            for i, (_, init) in enumerate(built_):
                b.set_initial(i, init)
            if tune:
                b.autotune(repeats=3)
            b.advance(5)
            assert b.synchronize() == 0
            return [b.download(i) for i in range(2)]
        finally:
            b.close()

    for a, c in zip(run(False), run(True)):
        assert np.array_equal(a, c)


@pytest.mark.gpu
@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_limiter_detector_forms_agree(built, order, precision):
    """The staged and compact KXRCF detectors, each under the barrier and the queue schedule and
    on either wave-kernel grid, flag the same cells, limit a perturbed state identically and give
    the same time steps."""
    mesh, init = instance_mesh(Instance(40, 20, 0.8, 1.25, order))
    rng = np.random.default_rng(order)
    out = []
    for staged, queue, one_per_sm in ((False, False, False), (True, False, False), (False, True, False),
                                      (True, True, False), (False, False, True), (True, True, True)):
        s = build_solver(mesh, order, 1.4, 0.1, 1.0e30, 6, precision=precision)
        try:
            sd, td = s.spatial_disc, s.temporal_disc
            sd.set_limiter_detector(staged)
            sd.set_limiter_schedule(queue)
            sd.set_limiter_grid(one_per_sm)
            assert sd.launch_config["limiter_grid"] == ("one_per_sm" if one_per_sm else "full")
            assert sd.launch_config["limiter_detector"] == ("staged" if staged else "compact")
            assert sd.launch_config["limiter_schedule"] == ("queue" if queue else "barrier")
            td.set_initial_on_device(init)
            U = sd.new_state()
            td.download(U)
            if not out:
                noise = 0.1 * rng.standard_normal(U[:, :, 1:].shape) * np.abs(U[:, :, :1])
            Up = U.copy()
            Up[:, :, 1:] += noise
            n_limited = sd.apply_limiter(Up)
            td.advance(6)
            td.synchronize()
            td.download(U)
            out.append((Up, n_limited, U, td.current_time))
        finally:
            s.close()
    La, na, Ua, ta = out[0]
    assert na > 0
    for Lb, nb, Ub, tb in out[1:]:
        assert na == nb
        assert np.array_equal(La, Lb)
        assert ta == tb and np.array_equal(Ua, Ub)


@pytest.mark.gpu
def test_limiter_schedule_switch_keeps_results(built):
    """Limiting under the barrier schedule, then switching the same context to the queue schedule
    (whose worklist must start empty) gives the results of a context that used only the queue."""
    mesh, init = instance_mesh(Instance(48, 24, 0.8, 1.25, 2))
    rng = np.random.default_rng(11)
    out = []
    for switch in (False, True):
        s = build_solver(mesh, 2, 1.4, 0.1, 1.0e30, 10, precision="fp64")
        try:
            sd, td = s.spatial_disc, s.temporal_disc
            td.set_initial_on_device(init)
            U = sd.new_state()
            td.download(U)
            if not out:
                noise = 0.1 * rng.standard_normal(U[:, :, 1:].shape) * np.abs(U[:, :, :1])
            Up = U.copy()
            Up[:, :, 1:] += noise
            if switch:
                sd.set_limiter_schedule(False)
                assert sd.apply_limiter(Up.copy()) > 0  # leaves worklist entries behind
            sd.set_limiter_schedule(True)
            n_limited = sd.apply_limiter(Up)
            td.advance(5)
            td.synchronize()
            td.download(U)
            out.append((Up, n_limited, U))
        finally:
            s.close()
    (La, na, Ua), (Lb, nb, Ub) = out
    assert na == nb and na > 0
    assert np.array_equal(La, Lb) and np.array_equal(Ua, Ub)
