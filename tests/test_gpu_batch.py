"""Batches: many ensembles in one persistent launch per step must give each
ensemble exactly the result it gets alone (same kernels, same summation
order), whatever else is in the batch and whenever it joined."""
import numpy as np
import pytest

from quest_b200 import capi, inputs as I

pytestmark = pytest.mark.gpu


def ensemble(seed, n, side, steps, amp):
    dots = I.make_dots(n, side, seed, omega_sigma=0.5, dipole=None, dipole_magnitude=2e-4)
    pulse = I.make_pulse(amplitude=amp, delay=0.05)
    return dots, pulse, I.Constants(num_timesteps=steps)


def solo(d, p, c, weights, steps):
    with capi.Simulation(d, p, c, weights=weights) as sim:
        sim.run(steps, record=False)
        return sim.state(), sim.bad_step()


def test_batch_equals_solo_runs(golden_weights):
    specs = [(11, 64, 0.05, 160, 5.0), (12, 200, 0.1, 96, 20.0), (13, 1000, 0.2, 160, 15.0)]
    ens = [ensemble(*s) for s in specs]
    batch = capi.Batch(8)
    sims = [capi.Simulation(d, p, c, weights=golden_weights) for d, p, c in ens]
    for s in sims:
        batch.add(s)
    assert batch.size()[0] == 3
    batch.run(10)  # 160 steps; the second member stops at its 96
    for (d, p, c), sim, spec in zip(ens, sims, specs):
        assert sim.next_step == spec[3]
        ref, bad = solo(d, p, c, golden_weights, spec[3])
        np.testing.assert_array_equal(sim.state(), ref)
        assert sim.bad_step() == bad == -1
    for s in sims:
        batch.remove(s)
        s.close()
    batch.close()


def test_member_joining_later_is_unaffected(golden_weights):
    a = ensemble(21, 300, 0.1, 128, 10.0)
    b = ensemble(22, 500, 0.15, 64, 25.0)
    batch = capi.Batch(4)
    sa = capi.Simulation(*a, weights=golden_weights)
    sb = capi.Simulation(*b, weights=golden_weights)
    batch.add(sa)
    batch.run(4)            # a alone: steps 0..63
    batch.add(sb)
    batch.run(4)            # a: 64..127, b: 0..63 together
    np.testing.assert_array_equal(sa.state(), solo(*a, golden_weights, 128)[0])
    np.testing.assert_array_equal(sb.state(), solo(*b, golden_weights, 64)[0])
    batch.close()
    sa.close()
    sb.close()


def test_batch_rejects_mismatched_members(golden_weights):
    a = ensemble(31, 100, 0.1, 64, 10.0)
    b = ensemble(32, 100, 0.1, 64, 10.0)
    b[2].interpolation_order = 3
    batch = capi.Batch(2)
    sa = capi.Simulation(*a, weights=golden_weights)
    sb = capi.Simulation(*b, weights=golden_weights)
    batch.add(sa)
    with pytest.raises(capi.QuestError):
        batch.add(sb)
    sc = capi.Simulation(*ensemble(33, 100, 0.1, 64, 10.0), weights=golden_weights)
    sc.run(5, record=False)
    with pytest.raises(capi.QuestError):
        batch.add(sc)  # not on a 16-step boundary
    batch.close()


def test_member_going_nonfinite_is_reported_and_the_others_are_unchanged(golden_weights):
    """The N = 200 workload with the pulse at delay 0.5 and dipoles 2e-3
    overflows (the reference's domain_error) near step 800; in a batch its
    first bad step is the one it has alone, read after every batch run, and
    the stable members beside it are bitwise their solo runs."""
    bad_wl = I.plain_small(n=200, steps=880, pulse_delay=0.5)
    with capi.Simulation(bad_wl.dots, bad_wl.pulse, bad_wl.constants, weights=golden_weights) as sim:
        with pytest.raises(capi.NonFiniteError) as e:
            sim.run(880, record=False)
    solo_bad = e.value.step
    assert 700 < solo_bad < 880
    good = [ensemble(21, 150, 0.1, 880, 10.0), ensemble(22, 300, 0.15, 880, 25.0)]
    batch = capi.Batch(4)
    sims = [capi.Simulation(bad_wl.dots, bad_wl.pulse, bad_wl.constants, weights=golden_weights)]
    sims += [capi.Simulation(d, p, c, weights=golden_weights) for d, p, c in good]
    for s in sims:
        batch.add(s)
    seen = None
    for blk in range(880 // 16):
        batch.run(1)
        if seen is None and sims[0].bad_step() >= 0:
            seen = (blk, sims[0].bad_step())
    assert seen is not None and seen[1] == solo_bad
    assert seen[0] == solo_bad // 16  # visible after the block that holds it
    for (d, p, c), sim in zip(good, sims[1:]):
        ref, bad = solo(d, p, c, golden_weights, 880)
        np.testing.assert_array_equal(sim.state(), ref)
        assert sim.bad_step() == bad == -1
    for s in sims:
        batch.remove(s)
        s.close()


@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_MIXED])
def test_batch_kernel_options_keep_the_bits(golden_weights, precision):
    """far_packed (packed FP32 pairs), far_gmajor (source-group-major task
    order) and mid_pipe (mid entries fetched several at a time) change how the
    batch's kernels run, not what they sum."""
    specs = [(31, 70, 0.05, 96, 5.0), (32, 400, 0.04, 96, 20.0), (33, 900, 0.2, 96, 15.0)]
    states = []
    for opts in ({}, {"far_packed": 1}, {"far_gmajor": 1}, {"far_packed": 1, "far_gmajor": 1, "mid_pipe": 1}):
        batch = capi.Batch(4)
        sims = [capi.Simulation(*ensemble(*s), weights=golden_weights, precision=precision) for s in specs]
        for s in sims:
            batch.add(s)
        for k, v in opts.items():
            batch.set_option(k, v)
        batch.run(6)
        states.append([s.state() for s in sims])
        for s in sims:
            batch.remove(s)
            s.close()
        batch.close()
    for other in states[1:]:
        for a, b in zip(states[0], other):
            np.testing.assert_array_equal(a, b)


def test_batch_autotuner_times_the_far_forms_and_keeps_the_bits(golden_weights):
    """The batch's first run times its far launch's forms (packed x task
    order); the tuned batch's members are still bitwise their solo runs."""
    specs = [(41, 300, 0.1, 64, 5.0), (42, 800, 0.15, 64, 20.0)]
    ens = [ensemble(*s) for s in specs]
    batch = capi.Batch(4)
    sims = [capi.Simulation(d, p, c, weights=golden_weights, precision=capi.PREC_MIXED) for d, p, c in ens]
    for s in sims:
        batch.add(s)
    batch.run(4)
    assert batch.get_option("tuned_far_us") > 0
    assert batch.get_option("far_packed") in (0, 1) and batch.get_option("far_gmajor") in (0, 1)
    for (d, p, c), sim in zip(ens, sims):
        with capi.Simulation(d, p, c, weights=golden_weights, precision=capi.PREC_MIXED) as solo_sim:
            solo_sim.run(64, record=False)
            np.testing.assert_array_equal(sim.state(), solo_sim.state())
    for s in sims:
        batch.remove(s)
        s.close()
    batch.close()


def test_batch_group_search_per_size_class(golden_weights):
    """"tune_group" times source tiles per far warp for each size class of
    members; each member then equals a solo run with its class's group set
    by hand."""
    specs = [(51, 100, 0.08, 64, 5.0), (52, 700, 0.15, 64, 20.0), (53, 2500, 0.25, 64, 10.0)]
    ens = [ensemble(*s) for s in specs]
    batch = capi.Batch(4)
    batch.set_option("tune_group", 1)
    sims = [capi.Simulation(d, p, c, weights=golden_weights, precision=capi.PREC_MIXED) for d, p, c in ens]
    for s in sims:
        batch.add(s)
    batch.run(4)
    assert batch.get_option("tune_group") == 1
    # 0: the members' own group was the fastest for that class
    classes = [batch.get_option(f"far_group_class{c}") for c in range(4)]
    assert all(g in (0, 1, 2, 4, 8) for g in classes)
    for (d, p, c), sim in zip(ens, sims):
        g = sim.get_option("far_group")
        assert g in (1, 2, 4, 8) and (g in classes or 0 in classes)
        with capi.Simulation(d, p, c, weights=golden_weights, precision=capi.PREC_MIXED) as solo_sim:
            solo_sim.set_option("far_group", g)
            solo_sim.run(64, record=False)
            np.testing.assert_array_equal(sim.state(), solo_sim.state())
    for s in sims:
        batch.remove(s)
        s.close()
    batch.close()
