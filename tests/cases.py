"""Parameter sets shared by the CPU and GPU parity tests.

Sizes are small enough for the FP64 oracle to finish in seconds; every case
puts the pulse through the TFSF box, the dispersive particle and the DFT
planes within the stepped window.
"""
from ref_cases import BASE

# 34^3 total grid (21 interior + 2*6 CPML + 1) with a thinner TFSF inset and
# box offset than the reference's 10/5, and a shorter pulse, so fields are
# non-trivial after a few hundred steps.  "sphere_ref" keeps the reference's
# constants on a 52^3 grid.
SMALL = dict(BASE, NCELLX=21, NCELLY=21, NCELLZ=21, NcpmlX=6, NcpmlY=6, NcpmlZ=6,
             tfsf_inset=4, box_offset=2, nano_sphere_radius=8e-9,
             BandWidth=8e15, lam_0=450e-9, Tend=420, NUM_freq=9)

CASES = {
    "vacuum": dict(SMALL, nano_sphere=0),
    "sphere_au": dict(SMALL),
    "cube_ag": dict(SMALL, nano_sphere=3, material=2, NCELLX=23, NCELLY=21, NCELLZ=25,
                    NcpmlX=5, NcpmlY=6, NcpmlZ=7, WL_or_freq=0),
    "sphere_ref": dict(BASE, NCELLX=31, NCELLY=31, NCELLZ=31, nano_sphere_radius=8e-9,
                       BandWidth=8e15, lam_0=450e-9, Tend=420, NUM_freq=9),
    "hydro": dict(SMALL, NONLOCAL=3, nano_sphere_radius=10e-9),
    "xpol": dict(SMALL, inc_phi_deg=90.0),
    "slab": dict(SMALL, nano_sphere=0, inf_disp_slab=2, dispersive_slab=2,
                 nano_sphere_radius=6e-9),
    "fixes": dict(SMALL, fixes=7),
    "dimer": dict(SMALL, geometry=1, axis=0, rod_length=8e-9, rod_diameter=4e-9, gap=2e-9,
                  NCELLX=25, inc_phi_deg=90.0),
    # 97 x 89 x 93 cells: large enough for the CPML-free interior box of pass
    # tiles (the smaller cases have CPML edge tiles only)
    "sphere_big": dict(SMALL, NCELLX=84, NCELLY=76, NCELLZ=80, nano_sphere_radius=12e-9),
    # 2x2 gold disks on a dielectric slab (eps 2.25)
    "disks_slab": dict(SMALL, geometry=2, disk_diameter=8e-9, disk_height=4e-9, pitch=12e-9,
                       disk_nx=2, disk_ny=2, slab_eps=2.25, slab_thickness=6e-9),
}


def make(mod, name, **over):
    kw = dict(CASES[name])
    kw.update(over)
    return mod.default_params(**kw)
