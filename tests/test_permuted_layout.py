"""The oracle on a node order like MIND.jl's DHS layout (children before parents, cells
interleaved round by round; src/model/micro/model.jl:906-1077): the same network in
discretization order gives the same raster and voltages within 1e-9 mV (only the order
of sums over siblings and co-located synapses changes)."""
import numpy as np

import mind_b200 as mb
import netcases
import oracle


def test_dhs_order_is_a_permutation_with_children_first():
    layout = mb.build(netcases.recurrent_trees(n_cells=6, synapses=8))
    order = netcases.dhs_order(layout, lanes=4)
    assert sorted(order.tolist()) == list(range(1, layout.n_nodes + 1))
    perm, new_of = netcases.permute_layout(layout, order)
    child = np.arange(1, perm.n_nodes + 1)
    has_parent = perm.parent > 0
    assert np.all(perm.parent[has_parent] > child[has_parent])


def test_oracle_on_dhs_order_matches_discretization_order():
    model = netcases.recurrent_trees(n_cells=12, synapses=16)
    layout = mb.build(model)
    perm, new_of = netcases.permute_layout(layout, netcases.dhs_order(layout, lanes=8))
    nodes = netcases.soma_nodes(layout)
    a = oracle.run(layout, 1200, nodes)
    b = oracle.run(perm, 1200, [int(new_of[n]) for n in nodes])
    assert a.status == 0 and b.status == 0
    assert np.max(np.abs(a.trace - b.trace)) <= 1e-9
    np.testing.assert_array_equal(a.spike_sids, b.spike_sids)
    np.testing.assert_array_equal(a.spike_times, b.spike_times)
    assert np.sum(a.spike_sids < layout.n_cells) > 5
