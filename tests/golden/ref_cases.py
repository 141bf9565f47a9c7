"""Parity cases run through the unmodified reference program.

Each case is an Input.txt deck (41 positional values, setup.cu:17-58) plus
the reference's hard-coded constants.  ``make_ref_golden.sh`` runs
oracle/_ref/fdtd_ref on a B200 for every case; ``import_ref_golden.py``
turns its text outputs (ScatAbs.<t>.txt, OUT.txt) into the .npz fixtures
under tests/golden/.  The same dicts build the oracle's and the product's
parameters in the tests.
"""

# Input.txt order (setup.cu:17-58) with the labels written to the deck.
INPUT_ORDER = [
    ("Tend", "d"), ("dx", "g"), ("dy", "g"), ("dz", "g"), ("num_trials", "d"),
    ("min_trials", "d"), ("max_trials", "d"), ("TE_TM", "d"), ("NCELLX", "d"),
    ("NCELLY", "d"), ("NCELLZ", "d"), ("NcpmlX", "d"), ("NcpmlY", "d"),
    ("NcpmlZ", "d"), ("inf_disp_slab", "d"), ("nano_sphere", "d"),
    ("nano_sphere_radius", "g"), ("material", "d"), ("first_medium", "d"),
    ("inc_plane", "d"), ("dispersive_slab", "d"), ("NUM_freq", "d"),
    ("WL_or_freq", "d"), ("NUM_freq_inc", "d"), ("Tend_inc", "d"), ("Snap_in", "d"),
    ("Freq_start", "d"), ("Test_offset", "d"), ("Spect_loc", "d"),
    ("BandWidth", "g"), ("NONLOCAL", "d"), ("Diverge_Gradient", "d"),
    ("t_skip", "d"), ("x_skip", "d"), ("y_skip", "d"), ("z_skip", "d"),
    ("Nonlocalend", "g"), ("MAX_AMP", "g"), ("TimeFactor", "g"), ("lam_0", "g"),
    ("StaticField", "d"),
]

BASE = dict(
    Tend=1000, dx=2e-9, dy=2e-9, dz=2e-9, num_trials=1, min_trials=1, max_trials=1,
    TE_TM=0, NCELLX=43, NCELLY=43, NCELLZ=43, NcpmlX=10, NcpmlY=10, NcpmlZ=10,
    inf_disp_slab=0, nano_sphere=1, nano_sphere_radius=10e-9, material=3,
    first_medium=1, inc_plane=0, dispersive_slab=0, NUM_freq=21, WL_or_freq=1,
    NUM_freq_inc=1, Tend_inc=1, Snap_in=0, Freq_start=0, Test_offset=0,
    Spect_loc=0, BandWidth=3e15, NONLOCAL=0, Diverge_Gradient=0, t_skip=1,
    x_skip=1, y_skip=1, z_skip=1, Nonlocalend=0.0, MAX_AMP=1.0, TimeFactor=1.0,
    lam_0=450e-9, StaticField=0,
)

CASES = {
    # 64^3 total, Au sphere r = 10 nm (5 cells), Drude+2CP, 1000 steps
    "sphere64": dict(BASE),
    # same grid, no particle: TFSF leakage / pure vacuum propagation
    "vacuum64": dict(BASE, nano_sphere=0, Tend=600),
    # hydrodynamic nonlocal model (NONLOCAL = 3), smaller run
    "hydro64": dict(BASE, NONLOCAL=3, Tend=600, nano_sphere_radius=12e-9),
    # silver cube (nano_sphere = 3), non-cubic grid, frequency grid
    "cube_ag": dict(BASE, nano_sphere=3, material=2, NCELLX=41, NCELLY=47, NCELLZ=45,
                    NcpmlX=8, NcpmlY=9, NcpmlZ=10, WL_or_freq=0, Tend=700, NUM_freq=17),
}


# Snapshot decks (Snap_in 3: aux lines and the |E| plane; Snap_in 2: the
# |P_d| and mean-density planes of the hydrodynamic model), with y/z skips
SNAP_CASES = {
    "snap_field": dict(BASE, Tend=400, Snap_in=3, t_skip=100, y_skip=2, z_skip=3),
    "snap_hydro": dict(BASE, NONLOCAL=3, Tend=400, nano_sphere_radius=12e-9, Snap_in=2, t_skip=100,
                       y_skip=1, z_skip=2),
}


def deck(case):
    """Input.txt text for a case dict."""
    lines = ["Input"]
    for name, kind in INPUT_ORDER:
        v = case[name]
        lines.append(f"{int(v)} {name}" if kind == "d" else f"{float(v)!r} {name}")
    return "\n".join(lines) + "\n"


if __name__ == "__main__":
    import os
    import sys
    out = sys.argv[1]
    which = sys.argv[2] if len(sys.argv) > 2 else "spectra"
    for name, case in (SNAP_CASES if which == "snap" else CASES).items():
        d = os.path.join(out, name)
        os.makedirs(d, exist_ok=True)
        with open(os.path.join(d, "Input.txt"), "w") as f:
            f.write(deck(case))
