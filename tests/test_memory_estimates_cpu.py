"""``getparam("memory_estimates")`` slot arithmetic (CPU): the reference's 16-slot layout
(memory_estimates, src/symbolic/maps.jl:307-356) filled from a plan's facts."""
from sdsb200.solver import memory_slots


def test_memory_slots_layout():
    n, ns, nb = 1000, 40, 3
    est = memory_slots("G", n, ns, nb, 8, factor_len=50_000, cb_len=20_000, device_bytes=5_000_000,
                       host_bytes=123_456, extra_device=1_000)
    assert len(est) == 16
    assert est[6] == 2 * 50_000 * 8 * nb                  # L and U^T panels
    assert est[7] == 2 * n * 8 * nb                       # D
    assert est[8] == 20_000 * 8 * nb                      # the update stack
    assert est[1] == 5_000_000 + 1_000                    # peak: every buffer, and the matching's
    assert est[0] == est[1] - est[8]                      # permanent: all but the update stack
    assert est[4] == est[1] and est[5] == 0               # no hybrid memory mode
    assert est[2] == est[3] == 123_456
    assert est[6] + est[7] + est[8] + est[9] + est[10] == 5_000_000
    assert est[11:] == [0] * 5
    spd = memory_slots("SPD", n, ns, 1, 4, factor_len=50_000, cb_len=0, device_bytes=2_000_000, host_bytes=0)
    assert spd[6] == 50_000 * 4 and spd[8] == 0 and spd[0] == spd[1] == 2_000_000
