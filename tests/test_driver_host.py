"""Host logic of the runMPMYDW driver: phase-1 termination (runMPMYDW.py:656-727)."""
from mpmwarpydw_b200.runMPMYDW import PhaseOneMonitor, load_domain
from mpmwarpydw_b200.utils.getArgs import defaults


def test_phase_one_runs_at_least_min_steps_then_stops_on_residual():
    m = PhaseOneMonitor(n_steps=5000, residual_threshold=1e-3, stall_threshold=-1.0, stall_steps=10**9, min_steps=1000)
    while m.running():
        assert m.update(10, residual=1e-6, mean_damage=0.0)
    assert m.counter == 1000 and not m.stopped_early


def test_phase_one_stops_at_n_steps():
    m = PhaseOneMonitor(n_steps=250, residual_threshold=1e-9, stall_threshold=-1.0, stall_steps=10**9)
    while m.running():
        m.update(25, residual=1.0, mean_damage=0.0)
    assert m.counter == 250


def test_damage_stall_ends_phase_after_the_stall_duration():
    m = PhaseOneMonitor(n_steps=10**6, residual_threshold=0.0, stall_threshold=1e-9, stall_steps=300, min_steps=1000)
    m.prev_damage = 0.0
    d, stopped_at = 0.0, None
    while m.running():
        d += 1e-3 if m.counter < 1500 else 0.0  # damage grows, then stalls
        if not m.update(1, residual=1.0, mean_damage=d):
            stopped_at = m.counter
            break
    assert m.stopped_early and stopped_at == 1500 + 300


def test_synthetic_domain_source():
    x, vol, props, over, d = load_domain("synthetic:block_collapse", defaults())
    assert x.shape == (64000, 3) and vol.shape == (64000,) and over["dt"] == 1e-4 and d is not None
