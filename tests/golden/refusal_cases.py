"""Invalid constructor inputs, shared by the generator of the reference's
refusals (``make_refusals.py``) and the test that replays them."""

import numpy as np

_D = [np.array([[0, 0, -5.0], [0, 0, 5.0]])]
_Y = [np.array([[0, 0, -5.0], [0, 0, 5.0]]), np.array([[1, 0, -5.0], [1, 0, 5.0]])]
_V = [np.array([[0, 0, 0.0], [1, 0, 1.0]]), np.array([[0, 0, 0.0], [-1, 0, 1.0]])]

REFUSALS = {
    "feed_wire_out_of_range": lambda: dict(wires=_D, feeds=[(2, None, 1.0)]),
    "feed_arclength_beyond_wire": lambda: dict(wires=_D, feeds=[(0, 50.0, 1.0)]),
    "feed_negative_arclength": lambda: dict(wires=_D, feeds=[(0, -1.0, 1.0)]),
    "degree_0": lambda: dict(wires=_D, degree=0),
    "degree_3": lambda: dict(wires=_D, degree=3),
    "nsegs_0": lambda: dict(wires=_D, nsegs=0),
    "radius_negative": lambda: dict(wires=_D, wire_radius=-1e-3),
    "radius_list_length": lambda: dict(wires=_Y, wire_radius=[1e-3]),
    "ground_eps_without_ground_z": lambda: dict(wires=_D, ground_eps=(13, 0.005)),
    "ground_model_unknown": lambda: dict(wires=_D, ground_z=-6.0, ground_eps=(13, 0.005), ground_model="bogus"),
    "ground_phi_mode_unknown": lambda: dict(wires=_D, ground_z=-6.0, ground_eps=(13, 0.005), ground_phi_mode="bogus"),
    "junction_port_out_of_range": lambda: dict(wires=_D, junction_ports=[0]),
    "junction_wire_out_of_range": lambda: dict(wires=_V, junctions=[[(0, "start"), (5, "start")]]),
    "junction_end_unknown": lambda: dict(wires=_V, junctions=[[(0, "start"), (1, "middle")]]),
    "node_gap_wire_out_of_range": lambda: dict(wires=_D, node_gaps=[(3, "start", 1.0)]),
    "edge_counts_per_wire": lambda: dict(wires=_D, n_per_edge_per_wire=[[5, 5]]),
    "feed_model_unknown": lambda: dict(wires=_D, feed_model="bogus"),
    "zero_length_wire": lambda: dict(wires=[np.array([[0, 0, 0.0], [0, 0, 0.0]])]),
    "conductivity_negative": lambda: dict(wires=_D, wire_conductivity=-1.0),
    "enrichment_variant_unknown": lambda: dict(wires=_D, enrichment_variant="bogus"),
    "enrichment_settings_with_enrichment_off": lambda: dict(wires=_D, n_qp_sing=16, enrichment_min_k=4,
                                                            enrichment_variant="stable", tikhonov_lambda=1e-2,
                                                            auto_tap_ratio_threshold=0.5),
    # singular enrichment: served alone, refused in three combinations
    "enrichment_on": lambda: dict(wires=_V, junctions=[[(0, "start"), (1, "start")]], use_singular_enrichment=True,
                                  enrichment_min_k=2),
    "enrichment_with_loading": lambda: dict(wires=_D, use_singular_enrichment=True, wire_conductivity=5.8e7),
    "enrichment_with_insulation": lambda: dict(wires=_D, use_singular_enrichment=True, insulation_radius=1e-3,
                                               insulation_eps_r=2.0),
    "enrichment_with_extended_kernel": lambda: dict(wires=_D, use_singular_enrichment=True, extended_kernel=True),
    "enrichment_with_per_wire_radius": lambda: dict(wires=_Y, use_singular_enrichment=True,
                                                    wire_radius=[1e-3, 2e-3]),
    "enrichment_with_equal_per_wire_radius": lambda: dict(wires=_Y, use_singular_enrichment=True,
                                                          wire_radius=[1e-3, 1e-3]),
    # the port and connection keywords, entry by entry
    "feeds_empty": lambda: dict(wires=_D, feeds=[]),
    "feeds_empty_with_junction_port": lambda: dict(wires=_V, junctions=[[(0, "start"), (1, "start")]], feeds=[],
                                                   junction_ports=[0]),
    "feed_arity": lambda: dict(wires=_D, feeds=[(0, None)]),
    "feed_second_entry_bad": lambda: dict(wires=_Y, feeds=[(0, None, 1.0), (1, None, 1.0, 0.0)]),
    "feed_wire_index_out_of_range": lambda: dict(wires=_D, feed_wire_index=3),
    "junction_group_empty": lambda: dict(wires=_V, junctions=[[(0, "start"), (1, "start")], []]),
    "junction_members_apart": lambda: dict(wires=_V, junctions=[[(0, "start"), (1, "end")]]),
    "junction_members_apart_third": lambda: dict(wires=_V + [np.array([[0, 0, 0.0], [0, 1, 1.0]])],
                                                 junctions=[[(0, "start"), (2, "start"), (1, "end")]]),
    "junction_port_listed_twice": lambda: dict(wires=_V, junctions=[[(0, "start"), (1, "start")]],
                                               junction_ports=[0, (0, 1.0)]),
    "node_gap_arity": lambda: dict(wires=_V, junctions=[[(0, "start"), (1, "start")]], node_gaps=[(0, "start")]),
    "node_gap_end_unknown": lambda: dict(wires=_V, junctions=[[(0, "start"), (1, "start")]],
                                         node_gaps=[(0, "middle", 1.0)]),
    "node_gap_not_at_junction": lambda: dict(wires=_V, junctions=[[(0, "start"), (1, "start")]],
                                             node_gaps=[(0, "end", 1.0)]),
    "node_gap_single_member": lambda: dict(wires=_V, junctions=[[(0, "start")]], node_gaps=[(0, "start", 1.0)]),
    "node_gap_member_twice": lambda: dict(wires=_V, junctions=[[(0, "start"), (1, "start")]],
                                          node_gaps=[(0, "start", 1.0), (0, "start", 1.0)]),
    "node_gap_junction_twice": lambda: dict(wires=_V, junctions=[[(0, "start"), (1, "start")]],
                                            node_gaps=[(0, "start", 1.0), (1, "start", 1.0)]),
    "node_gap_at_junction_port": lambda: dict(wires=_V, junctions=[[(0, "start"), (1, "start")]],
                                              junction_ports=[0], node_gaps=[(1, "start", 1.0)]),
    # refused at the solve, not by the constructor
    "pair_quadrature_0": lambda: dict(wires=_D, nsegs=21, wavelength=21.0, n_qp_pair=0),
    "pair_quadrature_9": lambda: dict(wires=_D, nsegs=21, wavelength=21.0, n_qp_pair=9),
    "wire_below_ground": lambda: dict(wires=_Y, nsegs=21, wavelength=21.0, ground_z=0.0),
    "edge_in_ground_plane": lambda: dict(wires=[np.array([[0, 0, 0.0], [1, 0, 0.0], [1, 0, 2.0]])], nsegs=11,
                                         wavelength=21.0, ground_z=0.0),
    "grounded_junction_port": lambda: dict(wires=_V, nsegs=11, wavelength=21.0, ground_z=0.0,
                                           junctions=[[(0, "start"), (1, "start")]], junction_ports=[0]),
    "second_junction_port_grounded": lambda: dict(
        wires=_V + [np.array([[0, 0, 2.0], [0, 0, 1.0]]), np.array([[0, 0, 2.0], [0, 1, 3.0]])], nsegs=11,
        wavelength=21.0, ground_z=0.0, junctions=[[(2, "start"), (3, "start")], [(0, "start"), (1, "start")]],
        junction_ports=[0, 1]),
}
AT_SOLVE = {"pair_quadrature_0", "pair_quadrature_9", "wire_below_ground", "edge_in_ground_plane",
            "grounded_junction_port", "second_junction_port_grounded"}
