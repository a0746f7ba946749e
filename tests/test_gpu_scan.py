"""Parameter scan (independent XXZ chains solved concurrently, one context and
stream per worker): concurrent and sequential runs give the same energies, and
each instance matches the FP64 CPU oracle run with the same seed and schedule
(fixed D, 1e-10 per site)."""
import pytest


@pytest.fixture(scope="module")
def T():
    import tensornetworks_b200 as T
    return T


@pytest.mark.gpu
def test_scan_concurrent_matches_sequential_and_oracle(T, oracle):
    from tensornetworks_b200 import scan
    inst = scan.make_xxz_scan(6, seed=5, Lmin=10, Lmax=16, Ds=(8, 16))
    opts = T.SolverOptions(precision=T.FP64)
    seq, t_seq = scan.run_scan(inst, workers=1, options=opts, sweeps=4, dstart=64)
    par, t_par = scan.run_scan(inst, workers=3, options=opts, sweeps=4, dstart=64)
    print("sequential", t_seq, "concurrent", t_par)
    for a, b in zip(seq, par):
        assert abs(a.energy_per_site - b.energy_per_site) < 1e-12
    assert len({r.worker for r in par}) > 1
    for r in seq:
        i = r.instance
        ref = oracle.find_ground_state(i.L, 0.5, i.D, [(4, i.D, i.D, 1e-12, 1e-12, 1e-10)], Jxy=i.Jxy, Jz=i.Jz,
                                       hz=-i.hz, seed=i.seed, eig_mode=1, gauge=1)
        assert abs(r.energy_per_site - ref["energy"] / i.L) < 1e-10, (i, r.energy_per_site, ref["energy"] / i.L)


def test_scan_instances_follow_the_plan():
    from tensornetworks_b200 import scan
    inst = scan.make_xxz_scan(64, seed=777)
    assert len(inst) == 64
    assert all(32 <= i.L <= 96 and i.D in (32, 64, 128) and -0.5 <= i.Jz <= 1.5 and 0 <= i.hz <= 0.5 for i in inst)
    assert scan.schedule_lines(128) == [(2, 16, 16), (2, 32, 16), (2, 64, 32), (2, 128, 64)]
