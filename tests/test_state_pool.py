"""step()'s pool of output states (lcode3d_b200.lcode._StatePool): an
entry is handed out again only when nothing outside the pool refers to the
state object or to any of its arrays. Host logic only (CPU tensors)."""
import torch

from lcode3d_b200 import lcode


def take(pool):
    return pool.take((3, 3), (5, 5), torch.device('cpu'))[0]


def test_dropped_state_is_reused_held_state_is_not():
    pool = lcode._StatePool()
    s0 = take(pool)
    s1 = take(pool)
    assert s1 is not s0
    s2 = take(pool)               # s0 and s1 are still held
    assert s2 is not s0 and s2 is not s1
    del s0
    s3 = take(pool)               # the reference loop's state before last
    assert s3 is pool.entries[0][0]
    assert s3 is not s1 and s3 is not s2


def test_a_held_array_keeps_its_state():
    pool = lcode._StatePool()
    s0 = take(pool)
    ez = s0.Ez                    # the caller keeps one array of the state
    first = id(s0)
    del s0
    for _ in range(2 * lcode._StatePool.SIZE):
        s = take(pool)
        assert id(s) != first or s.Ez is not ez
    assert pool.entries[0][1][7] is ez   # still the caller's array, never handed out again


def test_the_reference_loop_cycles_through_two_entries():
    pool = lcode._StatePool()
    state = take(pool)
    seen = set()
    for _ in range(10):
        state = take(pool)        # state = step(..., state, ...): the old state is dropped after the call
        seen.add(id(state))
    assert len(seen) <= lcode._StatePool.SIZE
    assert len(pool.entries) <= lcode._StatePool.SIZE


def test_ptrs_of_knows_only_unmodified_pool_states():
    pool = lcode._StatePool()
    s0 = take(pool)
    assert pool.ptrs_of(s0) is pool.entries[0][2]
    s0.Ez = torch.zeros(5, 5, dtype=torch.float64)   # the caller swapped an array
    assert pool.ptrs_of(s0) is None

    class Other:
        pass
    assert pool.ptrs_of(Other()) is None


def test_a_held_view_keeps_its_state():
    # a 0-d view such as an Ez(0,0) history entry shares the state's memory
    # without touching the reference counts of the state or its arrays
    pool = lcode._StatePool()
    s0 = take(pool)
    s0.Ez.fill_(7.0)
    v = s0.Ez[2, 2]
    first = pool.entries[0]
    del s0
    for _ in range(2 * lcode._StatePool.SIZE):
        s = take(pool)
        assert s is not first[0]
        s.Ez.fill_(-1.0)         # what the next step would write
    assert float(v) == 7.0
    del v
    assert take(pool) is first[0]   # free again once the view is gone


def test_a_slice_of_another_array_keeps_its_state():
    pool = lcode._StatePool()
    s0 = take(pool)
    row = s0.x_offt[1]           # any array of the one allocation
    first = pool.entries[0]
    del s0
    assert take(pool) is not first[0]
    del row
    assert take(pool) is first[0]
