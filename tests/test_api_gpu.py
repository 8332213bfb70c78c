"""The drop-in Python objects (api.py), driven the way the reference's
pipeline drives its own (pipeline.py:317-353 construction, :554-564 loop
body, :645-738 frame end), against the float64 oracle on the same keyed
noise: positions within 1e-12 µm, identical species, counters and FLIM
stacks; and SimulationPipeline.run with per-step recording."""
import numpy as np
import pytest

from flim_microscopy_simulator_with_causal_inference_b200 import api
from flim_microscopy_simulator_with_causal_inference_b200 import params as PR
from flim_microscopy_simulator_with_causal_inference_b200.config import config_from_dict
from oracle import oracle as O
from tests import cases

pytestmark = pytest.mark.gpu


def _oracle(cfg, duty):
    st = api.ParticleState(cfg)
    dp, _, _ = PR.build_dyn_params(cfg, st.N)
    _, pd = PR.build_phot_params(cfg, st.N, int(st.has_dye.sum()), duty)
    sp, _ = PR.build_scope_params(cfg)
    return O.OracleSimulation(cfg, st, dp, pd, sp, duty)


@pytest.mark.parametrize("case", ["rich_small", "binding_regions"])
def test_dropin_objects_match_the_oracle(case):
    cfg = config_from_dict(cases.get(case))
    duty = min(1.0, cfg.scan.dwell_time / cfg.scan.frame_interval)
    st = api.ParticleState(cfg)
    ps = api.PhotonSimulator(cfg, st, scan_duty_fraction=duty, precision=64)
    dyn = api.DynamicsEngine(cfg, st, precision=64)
    vm = api.VirtualMicroscope(cfg, st, precision=64)
    orc = _oracle(cfg, duty)
    n_ph = 0
    for _ in range(25):
        dyn.step()
        batch = ps.evolve_one_bd_step()
        vm.process_photons(batch)
        ob = orc.bd_step()
        assert np.array_equal(np.asarray(batch.particle_idx[:batch.n_photons]), ob[0])
        n_ph += batch.n_photons
    assert n_ph > 0
    np.testing.assert_allclose(st.positions, orc.pos, rtol=0, atol=1e-12)
    assert np.array_equal(st.species_id, orc.species) and np.array_equal(st.is_alive.astype(np.uint8), orc.alive)
    c = orc.counters
    assert (dyn.n_catalytic, dyn.n_recruited, dyn.n_detached, dyn.n_converted, dyn.n_bindings, dyn.n_dissociations) \
        == (c[PR.C_CATALYTIC], c[PR.C_RECRUITED], c[PR.C_DETACHED], c[PR.C_CONVERTED], c[PR.C_BINDINGS],
            c[PR.C_DISSOC])
    frame = vm.finalize_frame()
    assert np.array_equal(frame.flim_stack, orc.finalize_frame())


def test_pipeline_run_with_subframe_recording():
    raw = cases.get("rich_small")
    raw["scan"]["n_frames"] = 2
    raw["simulation_time"] = 2 * raw["scan"]["frame_interval"]
    cfg = config_from_dict(raw)
    res = api.SimulationPipeline(cfg, record_subframe=True, precision=64).run()
    pipe = api.SimulationPipeline(cfg, record_subframe=False, precision=64)
    assert len(res.frames) == pipe.n_frames == 2
    sub = res.subframe_data
    assert isinstance(sub, api.SubFrameData)
    n = pipe.n_frames * pipe.n_bd_per_frame
    assert sub.n_catalytic.shape == (n,) and sub.steps_per_frame == pipe.n_bd_per_frame
    assert sub.dt_s == cfg.bd_timestep
    assert np.all((sub.mean_fret_E >= 0.0) & (sub.mean_fret_E <= 1.0))
    # per-step species counts add up to the alive particles of each step
    total_alive = sum(sub.species_counts[s.name] for s in cfg.species)
    assert np.all(total_alive > 0)
    # the same run without recording gives the same frames (keyed noise)
    res2 = pipe.run()
    for a, b in zip(res.frames, res2.frames):
        assert np.array_equal(a.flim_frame.flim_stack, b.flim_frame.flim_stack)
    # per-step photon counts add up to the run's emitted photons
    assert int(sub.total_photons.sum()) == res.total_photons_emitted
    assert int(sub.n_bindings.sum()) == res.total_bindings
