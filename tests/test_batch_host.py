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
