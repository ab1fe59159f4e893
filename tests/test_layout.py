"""Host-side packing (build) invariants, mirroring pack_micro (CPU)."""
import numpy as np

import mind_b200 as mb
from mind_b200 import networks


def test_config1_layout_shape():
    layout = mb.build(networks.config1())
    assert layout.n_cells == 64
    assert layout.n_nodes == 64 * 54          # root + (1 seg + end) + (50 seg + end)
    assert layout.segment_count == 64 * 51
    assert [g.mechanism.name for g in layout.groups] == ["hh", "pas", "ExpSyn", "NetStim"]
    assert [g.rows for g in layout.groups] == [64, 3200, 640, 640]


def test_parents_first_and_axial_diagonal():
    layout = mb.build(networks.config1(n_cells=3))
    parent = layout.parent.astype(np.int64)
    idx = np.arange(1, layout.n_nodes + 1)
    assert np.all((parent == 0) | (parent < idx))
    expected = np.where(parent > 0, layout.axial, 0.0)
    for child in idx[parent > 0]:
        expected[parent[child - 1] - 1] += layout.axial[child - 1]
    np.testing.assert_array_equal(layout.axial_diagonal, expected)


def test_point_rows_sorted_by_node_and_logical_ids():
    layout = mb.build(networks.config1(n_cells=5))
    syn = layout.group("ExpSyn")
    assert np.all(np.diff(syn.nodes) >= 0)
    stim = layout.group("NetStim")
    assert np.all(stim.nodes == 0)
    # point logical id = point index + node count (micro/model.jl:510-530)
    first_stim_point = 5 * 10 + 1
    assert int(stim.logical_ids[0]) == first_stim_point + layout.n_nodes
    # every point maps back to its (group, row)
    for p in range(len(layout.point_group)):
        g = layout.groups[layout.point_group[p] - 1]
        assert 1 <= layout.point_row[p] <= g.rows


def test_fanout_csr_grouped_by_source():
    layout = mb.build(networks.config1(n_cells=2))
    off = layout.fanout_offsets
    assert off[0] == 1 and off[-1] == len(layout.edge_targets) + 1
    assert np.all(np.diff(off) >= 0)
    # NetStim sources (after the 2 detectors) each drive exactly one ExpSyn
    assert np.all(np.diff(off)[2:] == 1)
    assert np.all(np.diff(off)[:2] == 0)


def test_config2_and_config3_small_builds():
    l2 = mb.build(networks.config2(n_cells=12, synapses_per_cell=5))
    sizes = np.diff(l2.cell_offsets)
    assert l2.n_cells == 12
    seg_per_cell = [sum(len(v) - 1 for v in l2.morphologies[l2.cell_morphology[c]].section_nodes.values())
                    for c in range(12)]
    assert all(100 <= s <= 1000 for s in seg_per_cell)
    assert np.all(sizes > np.array(seg_per_cell))
    l3 = mb.build(networks.config3(n_cells=10, synapses_per_cell=20))
    assert [g.mechanism.name for g in l3.groups] == ["hh", "pas", "Exp2Syn", "NetStim", "IClamp"]
    hh_nodes = l3.group("hh").rows
    assert hh_nodes > 10   # soma plus the proximal 100 um sections
