"""Known-answer cases transcribed from the reference's own unit tests.

The reference (Rust) cannot be built or run here, so its test assertions are
the golden vectors.  Each case cites the test it comes from; values are the
asserted expectations (tolerances as in the reference test).
"""
import math

# ---------------------------------------------------------------------------
# Linear solves (src/solver/cpu.rs:187-397, src/sparse.rs:181-227,
# src/solver/sparse_direct.rs:67-86).  Matrices as (n, ncols, triplets).
# ---------------------------------------------------------------------------
REAL_SOLVES = [
    dict(name="identity_2x2", src="cpu.rs:189-197", n=2, ncols=2,
         trip=[(0, 0, 1.0), (1, 1, 1.0)], b=[3.0, 7.0], x=[3.0, 7.0], tol=1e-12),
    dict(name="known_2x2", src="cpu.rs:199-207", n=2, ncols=2,
         trip=[(0, 0, 2.0), (0, 1, 1.0), (1, 0, 5.0), (1, 1, 7.0)], b=[11.0, 13.0],
         x=[64.0 / 9.0, -29.0 / 9.0], tol=1e-12),
    dict(name="pivoting_3x3", src="cpu.rs:209-229", n=3, ncols=3,
         trip=[(0, 1, 2.0), (0, 2, 1.0), (1, 0, 1.0), (1, 1, 1.0), (1, 2, 1.0), (2, 0, 2.0),
               (2, 1, 1.0)], b=[5.0, 4.0, 4.0], x=[1.0, 2.0, 1.0], tol=1e-12),
    dict(name="one_by_one", src="cpu.rs:262-268", n=1, ncols=1, trip=[(0, 0, 5.0)], b=[15.0],
         x=[3.0], tol=1e-12),
    dict(name="tridiag_spmv_check", src="cpu.rs:368-396", n=3, ncols=3,
         trip=[(0, 0, 4.0), (0, 1, -1.0), (1, 0, -1.0), (1, 1, 4.0), (1, 2, -1.0), (2, 1, -1.0),
               (2, 2, 4.0)], b=[1.0, 5.0, 10.0], x=None, tol=1e-10),
    dict(name="sparse_lu_known_2x2", src="sparse_direct.rs:67-77", n=2, ncols=2,
         trip=[(0, 0, 2.0), (0, 1, 1.0), (1, 0, 5.0), (1, 1, 7.0)], b=[11.0, 13.0],
         x=[64.0 / 9.0, -29.0 / 9.0], tol=1e-10),
]

REAL_ERRORS = [
    dict(name="singular", src="cpu.rs:231-242", n=2, ncols=2,
         trip=[(0, 0, 1.0), (0, 1, 2.0), (1, 0, 2.0), (1, 1, 4.0)], b=[3.0, 6.0], err="singular"),
    dict(name="dimension_mismatch", src="cpu.rs:244-254", n=2, ncols=2,
         trip=[(0, 0, 1.0), (1, 1, 1.0)], b=[1.0, 2.0, 3.0], err="dimension"),
    dict(name="nonsquare", src="cpu.rs:256-260", n=2, ncols=3,
         trip=[(0, 0, 1.0), (1, 1, 1.0)], b=[1.0, 2.0], err="dimension"),
    dict(name="sparse_lu_singular", src="sparse_direct.rs:79-85", n=2, ncols=2,
         trip=[(0, 0, 1.0), (1, 0, 1.0)], b=[1.0, 1.0], err="singular"),
]

COMPLEX_SOLVES = [
    dict(name="c_identity_2x2", src="cpu.rs:281-291", n=2,
         trip=[(0, 0, 1 + 0j), (1, 1, 1 + 0j)], b=[3 + 1j, 7 - 2j], x=[3 + 1j, 7 - 2j], tol=1e-12),
    dict(name="c_known_2x2", src="cpu.rs:293-311", n=2,
         trip=[(0, 0, 1 + 1j), (0, 1, 2 + 0j), (1, 1, 1 - 1j)], b=[5 + 1j, 2 - 2j],
         x=[1 + 0j, 2 + 0j], tol=1e-12),
    dict(name="c_pivoting", src="cpu.rs:347-366", n=2,
         trip=[(0, 1, 1 + 1j), (1, 0, 1 + 0j), (1, 1, 2 + 0j)], b=[1 + 1j, 3 + 0j],
         x=[1 + 0j, 1 + 0j], tol=1e-12),
]
COMPLEX_ERRORS = [
    dict(name="c_singular", src="cpu.rs:313-331", n=2,
         trip=[(0, 0, 1 + 1j), (0, 1, 2 + 2j), (1, 0, 1 + 0j), (1, 1, 2 + 0j)], b=[1 + 0j, 1 + 0j]),
]

# CsrMatrix known answers (src/sparse.rs:181-227)
CSR_CASES = [
    dict(name="duplicates_summed", src="sparse.rs:200-206", n=2,
         trip=[(0, 0, 1.0), (0, 0, 2.0), (1, 1, 3.0)], dense=[[3.0, 0.0], [0.0, 3.0]], nnz=2),
    dict(name="identity", src="sparse.rs:191-198", n=2, trip=[(0, 0, 1.0), (1, 1, 1.0)],
         dense=[[1.0, 0.0], [0.0, 1.0]], nnz=2),
    dict(name="empty", src="sparse.rs:184-189", n=3, trip=[], dense=[[0.0] * 3] * 3, nnz=0,
         row_ptr=[0, 0, 0, 0]),
]
SPMV_CASES = [
    dict(name="spmv_2x2", src="sparse.rs:208-215", n=2, trip=[(0, 0, 2.0), (0, 1, 1.0), (1, 1, 3.0)],
         x=[1.0, 2.0], y=[4.0, 6.0]),
]

# ---------------------------------------------------------------------------
# MNA compiler (src/compiler.rs:772-1981).  Components use integer node labels
# with 0 = ground; the reference's string names "1", "2", ... map to 1, 2, ...
# Each component: (kind, name, nodes, value-or-params).
# Expected dense G entries are checked to 1e-9 as in the reference tests
# (so GMIN = 1e-12 on node diagonals is inside the tolerance).
# ---------------------------------------------------------------------------
DMOD = dict(is_=1e-14, n=1.0)
MNA_CASES = [
    dict(name="single_resistor_to_ground", src="compiler.rs:773-790",
         comps=[("R", "R1", (1, 0), 1000.0)], size=1, node_labels=[1], branches=[],
         g={(0, 0): 0.001}),
    dict(name="voltage_divider", src="compiler.rs:793-855",
         comps=[("V", "V1", (1, 0), 5.0), ("R", "R1", (1, 2), 1000.0), ("R", "R2", (2, 0), 1000.0)],
         size=3, node_labels=[1, 2], branches=["V1"],
         g={(0, 0): 0.001, (0, 1): -0.001, (0, 2): 1.0, (1, 0): -0.001, (1, 1): 0.002, (1, 2): 0.0,
            (2, 0): 1.0, (2, 1): 0.0, (2, 2): 0.0},
         b_dc=[0.0, 0.0, 5.0]),
    dict(name="rc_circuit", src="compiler.rs:858-912",
         comps=[("V", "V1", (1, 0), None, (1.0, 0.0)), ("R", "R1", (1, 2), 100.0),
                ("C", "C1", (2, 0), 1e-6)],
         size=3, g={(0, 0): 0.01, (0, 1): -0.01, (0, 2): 1.0, (1, 0): -0.01, (1, 1): 0.01, (2, 0): 1.0},
         c={(1, 1): 1e-6, (0, 0): 0.0, (0, 1): 0.0}, c_tol=1e-18, b_ac={2: 1 + 0j}),
    dict(name="inductor_stamps", src="compiler.rs:915-945",
         comps=[("L", "L1", (1, 2), 0.001)], size=3, branches=["L1"],
         g={(0, 2): 1.0, (2, 0): 1.0, (1, 2): -1.0, (2, 1): -1.0, (0, 0): 0.0, (1, 1): 0.0, (2, 2): 0.0},
         c={(2, 2): -0.001}, c_tol=1e-9),
    dict(name="current_source", src="compiler.rs:948-964",
         comps=[("I", "I1", (1, 0), 2.0)], size=1, b_dc=[-2.0]),
    dict(name="current_source_between_nodes", src="compiler.rs:967-988",
         comps=[("I", "I1", (1, 2), 3.0, (1.0, 90.0))], size=2, b_dc=[-3.0, 3.0],
         b_ac={0: -complex(math.cos(math.pi / 2), math.sin(math.pi / 2)),
               1: complex(math.cos(math.pi / 2), math.sin(math.pi / 2))}),
    dict(name="two_resistors_in_series", src="compiler.rs:1027-1057",
         comps=[("R", "R1", (1, 2), 100.0), ("R", "R2", (2, 0), 200.0)], size=2,
         g={(0, 0): 0.01, (0, 1): -0.01, (1, 0): -0.01, (1, 1): 0.015}),
    dict(name="parallel_resistors", src="compiler.rs:1242-1262",
         comps=[("R", "R1", (1, 0), 100.0), ("R", "R2", (1, 0), 200.0)], size=1, g={(0, 0): 0.015}),
    dict(name="empty_circuit", src="compiler.rs:1103-1111", comps=[], size=0),
]

DESCRIPTOR_CASES = [
    dict(name="single_diode", src="compiler.rs:1281-1333",
         comps=[("V", "V1", (1, 0), 1.0), ("D", "D1", (1, 0), DMOD)],
         diode=dict(anode=0, cathode="S", g_valid=[True, False, False, False], b_idx=[0, "S"],
                    is_val=1e-14, n_vt=0.02585)),
    dict(name="diode_between_non_ground", src="compiler.rs:1336-1397",
         comps=[("R", "R1", (1, 0), 1000.0), ("R", "R2", (2, 0), 1000.0),
                ("D", "D1", (1, 2), dict(is_=1e-14, n=1.5))],
         diode=dict(anode=0, cathode=1, g_valid=[True, True, True, True], b_idx=[0, 1],
                    is_val=1e-14, n_vt=1.5 * 0.02585),
         g={(0, 0): 0.001, (1, 1): 0.001, (0, 1): 0.0, (1, 0): 0.0}),
    dict(name="diode_ground_cathode", src="compiler.rs:1469-1506",
         comps=[("R", "R1", (1, 0), 1000.0), ("D", "D1", (1, 0), DMOD)],
         diode=dict(anode=0, cathode="S", g_valid=[True, False, False, False], b_idx=[0, "S"]),
         g_at_aa=0.001),
    dict(name="diode_ground_anode", src="compiler.rs:1509-1542",
         comps=[("R", "R1", (1, 0), 1000.0), ("D", "D1", (0, 1), DMOD)],
         diode=dict(anode="S", cathode=0, g_valid=[False, True, False, False], b_idx=["S", 0])),
    dict(name="single_bjt", src="compiler.rs:1593-1671",
         comps=[("V", "V1", (1, 0), 5.0), ("R", "R1", (1, 2), 10000.0), ("R", "R2", (1, 3), 1000.0),
                ("R", "R3", (4, 0), 100.0),
                ("Q", "Q1", (3, 2, 4), dict(is_=1e-14, bf=200.0, br=2.0, nf=1.0, nr=1.0, npn=True))],
         bjt=dict(collector=2, base=1, emitter=3, polarity=1.0, g_valid=[True] * 9, b_idx=[2, 1, 3],
                  is_val=1e-14, bf=200.0, br=2.0, nf_vt=0.02585, nr_vt=0.02585)),
    dict(name="bjt_to_ground", src="compiler.rs:1741-1800",
         comps=[("R", "R1", (1, 0), 1000.0), ("R", "R2", (2, 0), 1000.0),
                ("Q", "Q1", (1, 2, 0), dict(is_=1e-16, bf=100.0, br=1.0, nf=1.0, nr=1.0, npn=True))],
         bjt=dict(collector=0, base=1, emitter="S",
                  g_valid=[True, True, False, True, True, False, False, False, False],
                  b_idx=[0, 1, "S"])),
    dict(name="single_mosfet", src="compiler.rs:1674-1738",
         comps=[("V", "V1", (1, 0), 5.0), ("R", "R1", (1, 2), 1000.0), ("R", "R2", (3, 0), 100.0),
                ("M", "M1", (2, 1, 3), dict(vto=0.7, kp=1.1e-4, lam=0.04, nmos=True))],
         mosfet=dict(drain=1, gate=0, source=2, polarity=1.0, g_valid=[True] * 6, b_idx=[1, 2],
                     vto=0.7, kp=1.1e-4, lam=0.04)),
    dict(name="mosfet_to_ground", src="compiler.rs:1803-1854",
         comps=[("R", "R1", (1, 0), 1000.0), ("R", "R2", (2, 0), 1000.0),
                ("M", "M1", (1, 2, 0), dict(vto=1.0, kp=2e-5, lam=0.0, nmos=True))],
         mosfet=dict(drain=0, gate=1, source="S",
                     g_valid=[True, True, False, False, False, False], b_idx=[0, "S"])),
    dict(name="mixed_devices", src="compiler.rs:1901-1980",
         comps=[("V", "V1", (1, 0), 5.0), ("R", "R1", (1, 2), 1000.0), ("R", "R2", (3, 0), 1000.0),
                ("R", "R3", (4, 0), 1000.0), ("R", "R4", (5, 0), 1000.0), ("D", "D1", (2, 0), DMOD),
                ("Q", "Q1", (3, 2, 4), dict(is_=1e-16, bf=100.0, br=1.0, nf=1.0, nr=1.0, npn=True)),
                ("M", "M1", (3, 2, 5), dict(vto=0.7, kp=1.1e-4, lam=0.04, nmos=True))],
         counts=dict(diodes=1, bjts=1, mosfets=1, n_nodes=5, size=6)),
]

# End-to-end DC known answers (tests/integration_test.rs:48-131).
DC_CASES = [
    dict(name="voltage_divider_dc", src="integration_test.rs:48-84",
         comps=[("V", "V1", (1, 0), 10.0), ("R", "R1", (1, 2), 1000.0), ("R", "R2", (2, 0), 1000.0)],
         v={1: 10.0, 2: 5.0}, i={"V1": -0.005}, v_tol=1e-6, i_tol=1e-9),
    dict(name="current_source_dc", src="integration_test.rs:86-104",
         comps=[("I", "I1", (0, 1), 0.001), ("R", "R1", (1, 0), 1000.0)], v={1: 1.0}, v_tol=1e-9),
    dict(name="voltage_divider_unequal", src="integration_test.rs:106-125",
         comps=[("V", "V1", (1, 0), 10.0), ("R", "R1", (1, 2), 1000.0), ("R", "R2", (2, 0), 2000.0)],
         v={2: 20.0 / 3.0}, v_tol=1e-6),
]


def build_circuit(comps):
    """Turn a component list of these cases into an ohmnivore_b200 Circuit."""
    from ohmnivore_b200 import circuits as ck
    b = ck.CircuitBuilder()
    for c in comps:
        kind, name, nodes = c[0], c[1], c[2]
        val = c[3] if len(c) > 3 else None
        ac = c[4] if len(c) > 4 else None
        if kind == "R":
            b.resistors([nodes[0]], [nodes[1]], [val], names=[name])
        elif kind == "C":
            b.capacitors([nodes[0]], [nodes[1]], [val], names=[name])
        elif kind == "L":
            b.inductors([nodes[0]], [nodes[1]], [val], names=[name])
        elif kind == "V":
            b.vsource(nodes[0], nodes[1], dc=val, ac=ac, name=name)
        elif kind == "I":
            b.isource(nodes[0], nodes[1], dc=val, ac=ac, name=name)
        elif kind == "D":
            b.diodes([nodes[0]], nodes[1], is_=val["is_"], n=val["n"], names=[name])
        elif kind == "Q":
            b.bjts([nodes[0]], [nodes[1]], [nodes[2]], is_=val["is_"], bf=val["bf"], br=val["br"],
                   nf=val["nf"], nr=val["nr"], npn=val["npn"], names=[name])
        elif kind == "M":
            b.mosfets([nodes[0]], [nodes[1]], [nodes[2]], vto=val["vto"], kp=val["kp"], lam=val["lam"],
                      nmos=val["nmos"], names=[name])
    return b.build()
