"""Host side of the batched pressure-correction systems: every system comes from its
own generator, so a pool of processes makes the same inputs as one process."""
import numpy as np


def test_p_prime_host_is_the_same_in_a_process_pool():
    from kcfd.batch import p_prime_host, p_prime_sizes
    serial, s1 = p_prime_host(3, n_min=200, n_max=800, seed=5, workers=0)
    pooled, s2 = p_prime_host(3, n_min=200, n_max=800, seed=5, workers=2)
    np.testing.assert_array_equal(s1, s2)
    np.testing.assert_array_equal(s1, p_prime_sizes(3, 200, 800, 5))
    for a, b in zip(serial, pooled):
        pts_a, cells_a, bd_a, g_a, r_a = a
        pts_b, cells_b, bd_b, g_b, r_b = b
        np.testing.assert_array_equal(pts_a, pts_b)
        np.testing.assert_array_equal(cells_a, cells_b)
        np.testing.assert_array_equal(g_a, g_b)
        np.testing.assert_array_equal(r_a, r_b)
        assert sorted(bd_a) == sorted(bd_b)
        for k in bd_a:
            np.testing.assert_array_equal(np.asarray(bd_a[k]), np.asarray(bd_b[k]))


def test_lpt_shards_cover_every_system_once():
    from kcfd.batch import lpt_shards, p_prime_sizes
    sizes = p_prime_sizes(1024, 2000, 200000, 0)
    for world in (1, 2, 3, 8):
        shards = lpt_shards(sizes * 4, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(1024))
        loads = [sizes[s].sum() for s in shards]
        assert max(loads) - min(loads) <= sizes.max()


def test_graded_teams_follow_the_batch():
    """kcfd_batch_plan (host only, the rule kcfd_batch_create applies), on the C4 size
    distribution: a 128-system batch spreads its big systems over clusters of 8, 4 and 2
    CTAs (R = 8192 rows), the full 1,024 keeps all but the largest on one CTA (R = 65536:
    clusters of 2 from 131,072 rows) -- R is the smallest 8192 * 2^k whose cluster teams ask
    for at most 3.5 CTAs per SM."""
    from kcfd.batch import p_prime_sizes, plan_teams
    sizes = np.asarray(p_prime_sizes(1024, 2000, 200000, 0))
    t128 = plan_teams(sizes[:128])
    n = sizes[:128]
    assert ((t128 >= 2).sum(), (t128 == 1).sum(), (t128 == 0).sum()) == (75, 0, 53)
    np.testing.assert_array_equal(t128, np.where(n >= 8 * 8192, 8, np.where(n >= 4 * 8192, 4,
                                                                            np.where(n >= 2 * 8192, 2, 0))))
    t1024 = plan_teams(sizes)
    np.testing.assert_array_equal(t1024, np.where(sizes >= 131072, 2, np.where(sizes >= 16384, 1, 0)))

    def demand(n, R):
        q = n // R
        return int(np.where(q >= 8, 8, np.where(q >= 4, 4, np.where(q >= 2, 2, 0))).sum())
    assert demand(sizes, 32768) > 3.5 * 148 >= demand(sizes, 65536)
    assert demand(n, 8192) <= 3.5 * 148
    # one tier of 4 CTAs from 131,072 rows; no clusters at all
    t4 = plan_teams(sizes, cluster_size=4)
    np.testing.assert_array_equal(t4 == 4, sizes >= 131072)
    assert (plan_teams(sizes, cluster_rows=-1) <= 1).all()
