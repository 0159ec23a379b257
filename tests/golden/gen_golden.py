"""Generates the golden fixtures in this folder from the reference's OWN CPU code.

The reference (tacaswell/hipgisaxs) is C++; ``make -C oracle ref`` compiles its CPU hot-path
sources where they lie into ``oracle/_ref/libhigref.so``.  This script drives that library
through ``oracle/pyoracle.py`` (backend "ref") on small seeded cases and writes one .npz per
case: the inputs and the reference's outputs.  The tests check the plain-C oracle and the
CUDA path against these files, so parity stays pinned where the reference tree is absent.

Run from the repository root:  python tests/golden/gen_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import pyoracle as po  # noqa: E402


GRIDS = {
    "g16": dict(ncol=16, nrow=12, region=(-1.0, 0.0, 1.0, 2.0), ai=0.16, e=10.0, dn2=(0, 0)),
    "g16abs": dict(ncol=16, nrow=12, region=(-2.0, 0.0, 2.0, 3.0), ai=0.20, e=10.0,
                   dn2=(2 * 3e-6, 2 * 2e-8)),
}


def tri_case(rng, T, scale):
    sd = np.zeros((T, 8))
    sd[:, 0] = rng.uniform(0.2, 3.0, T)
    n = rng.normal(size=(T, 3))
    sd[:, 1:4] = n / np.linalg.norm(n, axis=1)[:, None]
    sd[:, 4:7] = rng.normal(scale=scale, size=(T, 3))
    return sd


def main():
    if not po.available("ref"):
        sys.exit("oracle/_ref/libhigref.so missing: run `make -C oracle ref` first")
    po.set_threads(4, "ref")
    rng = np.random.default_rng(20240601)
    out = {}
    # grids: a Born-like vacuum layer and a buried (absorbing) particle layer
    grids = GRIDS
    rots = {"id": np.eye(3),
            "r3": po.rot_mul(po.rot_mul(po.rot_axis(2, 0.35), po.rot_axis(0, 0.12)),
                             po.rot_axis(1, -0.2))}
    for gname, g in grids.items():
        G = po.Grid(g["ncol"], g["nrow"], *g["region"], g["ai"], g["e"], g["dn2"], backend="ref")
        base = dict(ncol=G.ncol, nrow=G.nrow, region=np.array(g["region"]), alpha_i_deg=g["ai"],
                    energy_kev=g["e"], dn2=np.array(g["dn2"], dtype=float), qx=G.qx, qy=G.qy,
                    qz=G.qz, alpha=G.alpha, qz_ext=G.qz_ext)
        np.savez_compressed(os.path.join(HERE, f"qgrid_{gname}.npz"), **base)
        # numeric form factor (approx triangle)
        for rname, R in rots.items():
            sd = tri_case(rng, 53, 6.0)
            ff = po.ff_approx_triangle(sd, G.qx, G.qy, G.qz_ext, R, "ref")
            np.savez_compressed(os.path.join(HERE, f"fftri_{gname}_{rname}.npz"), shape_def=sd,
                                rot=R, ff=ff, grid=gname)
        # analytic shapes
        shapes = {
            "cylinder": po.cylinder_params(5.0, 10.0, 0.05, 7),
            "sphere": [dict(type="radius", stat="gaussian", min=4, max=6, mean=5, deviation=0.3,
                            nvalues=5)],
            "box": [dict(type="xsize", stat="uniform", min=3, max=5, nvalues=3),
                    dict(type="ysize", min=4, max=4), dict(type="height", min=2, max=2)],
            "cube": [dict(type="height", stat="uniform", min=3, max=4, nvalues=2)],
            "prism3": [dict(type="edge", min=5, max=5), dict(type="height", min=3, max=3)],
            "prism6": [dict(type="edge", min=5, max=5), dict(type="height", min=3, max=3)],
            "pyramid": [dict(type="xsize", min=10, max=10), dict(type="ysize", min=10, max=10),
                        dict(type="height", min=3, max=3), dict(type="baseangle", min=60, max=60)],
        }
        for sname, params in shapes.items():
            ff = po.ff_analytic(G, sname, params, 0.1, 0.2, (1.0, 2.0, 3.0), rots["r3"])
            np.savez_compressed(os.path.join(HERE, f"ffana_{sname}_{gname}.npz"),
                                params=po.param_rows(params), tau=0.1, eta=0.2,
                                transvec=np.array([1.0, 2.0, 3.0]), rot=rots["r3"], ff=ff,
                                grid=gname)
        # lattice structure factor
        for lname, hkl, rep in (("hex", "100", [20, 20, 1]), ("cubic", "100", [5, 7, 3]),
                                ("fcc", "100", [4, 4, 4])):
            abc = np.array(po.lattice_vectors(lname, hkl)[:3])
            sf = po.sf_lattice(G, abc, rep, [20.0, 20.0, 20.0], (1.0, 2.0, 3.0), rots["r3"])
            np.savez_compressed(os.path.join(HERE, f"sf_{lname}_{gname}.npz"), abc=abc,
                                repet=np.array(rep, dtype=float), scaling=np.array([20.0] * 3),
                                center=np.array([1.0, 2.0, 3.0]), rot=rots["r3"], sf=sf,
                                grid=gname)
        # Fresnel / DWBA coefficients: substrate only, and a 3-layer stack
        for lname, layers, order in (
                ("sub", [(4.88e-6, 7.37e-8, 0.0, -1)], 0),
                ("stack", [(4.88e-6, 7.37e-8, 0.0, -1), (3e-6, 2e-8, 7.0, 1),
                           (1e-6, 1e-9, 3.0, 2)], 1)):
            fc = po.propagation_coeffs(G, layers, order)
            np.savez_compressed(os.path.join(HERE, f"fc_{lname}_{gname}.npz"),
                                layers=np.array(layers, dtype=float), order=order, fc=fc,
                                grid=gname)
    exact_fixtures()
    liquid_fixtures()
    smear_fixtures()
    print("golden fixtures written to", HERE)


def exact_fixtures():
    """The exact triangle form factor (NumericFormFactorC::compute_exact_triangle): a jittered
    80-face icosphere plus 20 random triangles, on both grids, unrotated and rotated."""
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from hipgisaxs_b200 import meshes
    rng = np.random.default_rng(20240605)
    V, F = meshes.icosphere(6.0, 1)
    V = V + rng.normal(scale=0.2, size=V.shape)
    tris = np.vstack([po.mesh_triangles(V, F), rng.normal(scale=5.0, size=(20, 9))])
    rots = {"id": np.eye(3),
            "r3": po.rot_mul(po.rot_mul(po.rot_axis(2, 0.35), po.rot_axis(0, 0.12)),
                             po.rot_axis(1, -0.2))}
    for gname in ("g16", "g16abs"):
        g = np.load(os.path.join(HERE, f"qgrid_{gname}.npz"))
        for rname, R in rots.items():
            ff = po.ff_exact_triangle(tris, g["qx"], g["qy"], g["qz_ext"], R, "ref")
            np.savez_compressed(os.path.join(HERE, f"ffexact_{gname}_{rname}.npz"), tris=tris,
                                rot=R, ff=ff, grid=gname)


LIQUID_CASES = {
    "para1d": ("para", (1, 3, 0.0, 12.0, 0.0, 2.0, 200.0)),
    "para2d_cubic": ("para", (2, 3, 10.0, 12.0, 1.5, 2.0, 300.0)),
    "para2d_hex": ("para", (2, 7, 10.0, 12.0, 1.5, 2.0, 300.0)),
    "py2d": ("py", (8.0, 0.3, 2)),
    "py3d": ("py", (8.0, 0.3, 3)),
}


def liquid_fixtures():
    """Paracrystal and Percus-Yevick structure factors (src/sf/liquid.cpp) on both grids."""
    for gname, g in GRIDS.items():
        G = po.Grid(g["ncol"], g["nrow"], *g["region"], g["ai"], g["e"], g["dn2"], backend="ref")
        for cname, (kind, args) in LIQUID_CASES.items():
            sf = po.sf_paracrystal(G, *args) if kind == "para" else po.sf_percus_yevick(G, *args)
            np.savez_compressed(os.path.join(HERE, f"sfliq_{cname}_{gname}.npz"), kind=kind,
                                args=np.array(args, dtype=float), sf=sf, grid=gname)


def smear_fixtures():
    """Convolutions::convolution_gaussian_2d on seeded images: narrow, wide (window larger than
    the image) and a non-square image."""
    rng = np.random.default_rng(20240606)
    for name, shape, sigma in (("s07", (12, 16), 0.7), ("s20", (12, 16), 2.0),
                               ("s35", (40, 48), 3.5)):
        img = rng.random(shape) * 1e3
        out = po.smear_gaussian(img, sigma, "ref")
        np.savez_compressed(os.path.join(HERE, f"smear_{name}.npz"), image=img, sigma=sigma,
                            smeared=out)


if __name__ == "__main__":
    if sys.argv[1:] == ["exact"]:
        po.set_threads(4, "ref")
        exact_fixtures()
    elif sys.argv[1:] == ["liquid"]:
        liquid_fixtures()
    elif sys.argv[1:] == ["smear"]:
        smear_fixtures()
    else:
        main()
