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

# Periodic x and y (periodic_xy): an 8 x 8 x 77 column with CPML in z only.
# "periodic_film" holds a 20 nm gold film (the reference's finite slab,
# inf_disp_slab = 2, thickness nano_sphere_radius); "periodic_spheres"
# puts a gold sphere on a 10 nm film in a 16 x 16 cell.
PERIODIC = dict(SMALL, nano_sphere=0, NCELLX=8, NCELLY=8, NCELLZ=60, NcpmlX=0, NcpmlY=0,
                NcpmlZ=8, tfsf_inset=8, periodic_xy=1, Tend=3000)
CASES.update({
    "periodic_vacuum": dict(PERIODIC),
    "periodic_film": dict(PERIODIC, inf_disp_slab=2, dispersive_slab=40, nano_sphere_radius=20e-9),
    "periodic_spheres": dict(PERIODIC, NCELLX=16, NCELLY=16, nano_sphere=1, inf_disp_slab=2,
                             dispersive_slab=40, nano_sphere_radius=10e-9, inc_phi_deg=30.0),
})


def gold_film_rt(lam, d):
    """R and T of a free-standing film of thickness d (m) at normal
    incidence from the Drude + two-critical-point gold permittivity the
    reference uses (setup.cu:1164-1211), by the Airy sums."""
    import numpy as np
    c0 = 2.99792458e8
    w = 2 * np.pi * c0 / np.asarray(lam)
    eps = 1.1431 - 1.3202e16 ** 2 / (w ** 2 + 1j * 1.0805e14 * w)
    for a, ph, om, ga in ((0.26698, -1.2371, 3.8711e15, 4.4642e14),
                          (3.0834, -1.0968, 4.1684e15, 2.3555e15)):
        eps = eps + a * om * (np.exp(1j * ph) / (om - w - 1j * ga) + np.exp(-1j * ph) / (om + w + 1j * ga))
    n = np.sqrt(eps)
    r12, r23 = (1 - n) / (1 + n), (n - 1) / (n + 1)
    e = np.exp(1j * n * w / c0 * d)
    den = 1 + r12 * r23 * e ** 2
    r = (r12 + r23 * e ** 2) / den
    t = (2 / (1 + n)) * (2 * n / (n + 1)) * e / den
    return np.abs(r) ** 2, np.abs(t) ** 2
