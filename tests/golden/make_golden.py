"""Regenerate the fixtures in tests/golden/ from the reference's own code.

Builds the checkers of oracle/build_ref.py (the reference's sources compiled
unmodified from the reference tree against the stand-in Eigen/boost headers
in oracle/refshim), runs them and packs their raw outputs:

  reference_tables.npz      TableKernel, BSpline / Wendland C4, Dim<3>
                            geometry, mapPositionThroughPlanes (ref_tables)
  reference_restart_<case>.npz  the reference's restart file (RestartRegistrar
                            ::dumpState through FlatFileIO, ascii) after a few
                            RK2 steps of one node set, and the state after
                            the reference restored that file
                            (RestartRegistrar::restoreState) and took more
                            steps (ref_sph --restart-dump / --restart-load)
  reference_sph_<case>.npz  one node set run through the reference's
                            SPHHydroBase / CRKSPHHydroBase, ConnectivityMap,
                            periodic boundaries and CheapSynchronousRK2
                            (ref_sph): the inputs, the ghosts and the
                            ConnectivityMap, every derivative field of one
                            evaluateDerivatives at t = 0, and the state after a
                            few RK2 steps

Needs the reference tree, so it runs in the development container only; the
committed .npz files are what the tests read.

    python tests/golden/make_golden.py [case ...]
"""
import hashlib
import importlib
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def _sod(gen, abi, nx, ny, nz, **kw):
    box = ((0.0, 0.0, 0.0), (1.0, ny / nx, nz / nx))
    ns = gen.sod(nx=nx, ny=ny, nz=nz, box=box, jitter=0.05)
    ns.vel[:, 0] = 0.05 * np.sin(2 * np.pi * ns.pos[:, 0])
    return ns, gen.sod_config(abi, ns_box=box, **kw)


def _kh(gen, abi, nx, ny, nz, **kw):
    box = ((0.0, 0.0, 0.0), (1.0, ny / nx, nz / nx))
    ns = gen.kelvin_helmholtz(nx=nx, ny=ny, nz=nz, box=box)
    return ns, gen.kh_config(abi, xmax=box[1], **kw)


def cases(pkg):
    """name -> (node set, config, RK2 steps).  Together they switch every
    option the device path implements at least once."""
    gen, abi = pkg.generators, pkg.abi
    c = {}
    c["sod"] = _sod(gen, abi, 16, 4, 4) + (3,)
    ns, cfg = _sod(gen, abi, 16, 4, 4, gradhCorrection=1, XSPH=1)
    c["sod_gradh_xsph"] = (ns, cfg, 3)
    ns, cfg = _sod(gen, abi, 16, 4, 4, densityUpdate=abi.DENSITY_INTEGRATE, HUpdate=abi.H_INTEGRATE,
                   epsTensile=0.3, nTensile=4.0, linearInExpansion=1, quadraticInExpansion=1)
    c["sod_integrate_tensile"] = (ns, cfg, 3)
    # the eigenvalue clamp of the bounded H policy: anisotropic, integrated H
    # with hmin and hmax inside the spread of its eigenvalues
    ns, cfg = _sod(gen, abi, 16, 4, 4, HUpdate=abi.H_INTEGRATE, hmin=0.06, hmax=0.09)
    rng = np.random.default_rng(7)
    ns.H[:, 0] *= rng.uniform(0.8, 1.3, ns.n)
    ns.H[:, 5] *= rng.uniform(1.0, 1.8, ns.n)
    ns.H[:, 1] = 0.15 * ns.H[:, 0] * rng.uniform(-1, 1, ns.n)
    ns.H[:, 4] = 0.15 * ns.H[:, 3] * rng.uniform(-1, 1, ns.n)
    c["sod_hclamp"] = (ns, cfg, 3)
    c["kh"] = _kh(gen, abi, 12, 12, 6) + (5,)
    # the Balsara shear correction of the Q (sheared flow: curl and div both nonzero)
    ns, cfg = _kh(gen, abi, 12, 12, 6, balsaraShearCorrection=1)
    c["kh_balsara"] = (ns, cfg, 5)
    ns, cfg = _kh(gen, abi, 12, 12, 6, compatibleEnergyEvolution=0, useVelocityMagnitudeForDt=1,
                  correctVelocityGradient=0)
    c["kh_noncompatible"] = (ns, cfg, 5)
    c["crk_sod"] = _sod(gen, abi, 16, 4, 4, hydro=abi.HYDRO_CRKSPH) + (3,)
    c["crk_kh"] = _kh(gen, abi, 12, 12, 6, hydro=abi.HYDRO_CRKSPH) + (5,)
    ns, cfg = _sod(gen, abi, 16, 4, 4, hydro=abi.HYDRO_CRKSPH, XSPH=1, crkVolumeType=abi.CRK_MASSOVERDENSITY)
    c["crk_sod_xsph_massoverdensity"] = (ns, cfg, 3)
    ns, cfg = _sod(gen, abi, 16, 4, 4, hydro=abi.HYDRO_CRKSPH, qType=abi.Q_CRKSPH_MONAGHAN_GINGOLD)
    c["crk_sod_crkq"] = (ns, cfg, 3)
    ns, cfg = _kh(gen, abi, 12, 12, 6, hydro=abi.HYDRO_CRKSPH, densityUpdate=abi.DENSITY_INTEGRATE,
                  crkVolumeType=abi.CRK_MASSOVERDENSITY)
    c["crk_kh_integrate_massoverdensity"] = (ns, cfg, 5)
    return c


def write_input(path, cfg, ns, nsteps):
    with open(path, "wb") as f:
        f.write(np.int64(ns.n).tobytes())
        f.write(np.int64(nsteps).tobytes())
        f.write(bytes(cfg))
        for a in (ns.pos, ns.vel, ns.mass, ns.rho, ns.eps, ns.H):
            f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())


def run_reference(exe, cfg, ns, nsteps):
    with tempfile.TemporaryDirectory() as td:
        for sub in ("eval", "steps"):
            os.makedirs(os.path.join(td, sub))
        write_input(os.path.join(td, "in.bin"), cfg, ns, nsteps)
        subprocess.check_call([exe, os.path.join(td, "in.bin"), td], stdout=subprocess.DEVNULL)
        out = {}
        for sub in ("", "eval", "steps"):
            d = os.path.join(td, sub)
            for f in sorted(os.listdir(d)):
                key = (sub + "/" if sub else "") + f[:-4]
                if f.endswith(".f64"):
                    out[key] = np.fromfile(os.path.join(d, f), dtype="<f8")
                elif f.endswith(".i64"):
                    out[key] = np.fromfile(os.path.join(d, f), dtype="<i8")
    return out


def sph_fixture(exe, name, ns, cfg, nsteps):
    r = run_reference(exe, cfg, ns, nsteps)
    data = {"input/config": np.frombuffer(bytes(cfg), dtype=np.uint8), "input/nsteps": np.int64(nsteps),
            "input/position": ns.pos, "input/velocity": ns.vel, "input/mass": ns.mass,
            "input/mass density": ns.rho, "input/specific thermal energy": ns.eps, "input/H": ns.H}
    for k, v in r.items():
        if k == "eval/pair accelerations":
            # Kept as a digest of the exact bytes (the array is 3 doubles per entry).
            data["eval/pair accelerations sha256"] = np.frombuffer(hashlib.sha256(v.tobytes()).digest(),
                                                                   dtype=np.uint8)
            data["eval/pair accelerations size"] = np.int64(v.size)
        elif k in ("conn_offsets", "conn_neighbors", "ghost_root"):
            data[k] = v.astype(np.int32)
        else:
            data[k] = v
    out = os.path.join(HERE, "reference_sph_%s.npz" % name)
    np.savez_compressed(out, **data)
    return out


def idealh_cases(pkg):
    """name -> (node set, config): Sod tubes whose H are perturbed away from
    the ideal (isotropic scale jitter; and with off-diagonal terms)."""
    gen, abi = pkg.generators, pkg.abi
    out = {}
    for name, aniso in (("iso", False), ("aniso", True)):
        box = ((0.0, 0.0, 0.0), (1.0, 0.25, 0.25))
        ns = gen.sod(nx=32, ny=8, nz=8, box=box, jitter=0.1, seed=3)
        rng = np.random.default_rng(1)
        ns.H[:, [0, 3, 5]] *= rng.uniform(0.6, 1.5, (ns.n, 1))
        if aniso:
            ns.H[:, 1] = 0.05 * ns.H[:, 0] * rng.uniform(-1, 1, ns.n)
            ns.H[:, 3] *= rng.uniform(0.8, 1.2, ns.n)
        out[name] = (ns, gen.sod_config(abi, ns_box=box))
    return out


def idealh_fixture(exe, name, ns, cfg, max_iterations=50, tolerance=1.0e-4):
    """The reference's iterateIdealH as its controller calls it: the relaxed
    H, the iteration count and the last maximum change it reports (printed
    to six significant digits by the reference)."""
    with tempfile.TemporaryDirectory() as td:
        os.makedirs(os.path.join(td, "idealh"))
        write_input(os.path.join(td, "in.bin"), cfg, ns, 0)
        subprocess.check_call([exe, "--ideal-h", str(max_iterations), repr(tolerance), os.path.join(td, "in.bin"), td],
                              stdout=subprocess.DEVNULL)
        H = np.fromfile(os.path.join(td, "idealh", "H.f64"), dtype="<f8")
        itd = np.fromfile(os.path.join(td, "idealh", "iterations_delta.f64"), dtype="<f8")
    data = {"input/config": np.frombuffer(bytes(cfg), dtype=np.uint8), "input/position": ns.pos,
            "input/velocity": ns.vel, "input/mass": ns.mass, "input/mass density": ns.rho,
            "input/specific thermal energy": ns.eps, "input/H": ns.H,
            "input/max_iterations": np.int64(max_iterations), "input/tolerance": np.float64(tolerance),
            "H": H, "iterations": np.int64(itd[0]), "max_delta_h_printed": np.float64(itd[1])}
    out = os.path.join(HERE, "reference_idealh_%s.npz" % name)
    np.savez_compressed(out, **data)
    return out


def restart_cases(pkg):
    """name -> (node set, config, steps before the dump, steps after the
    restore): SPH with compatible energy; SPH with grad-h, XSPH and no
    compatible energy; CRKSPH with the CRKSPH Q; CRKSPH with the
    Monaghan-Gingold Q."""
    gen, abi = pkg.generators, pkg.abi
    c = {}
    c["sph_kh"] = _kh(gen, abi, 8, 8, 4) + (2, 2)
    c["sph_sod_gradh_xsph_noncompatible"] = _sod(gen, abi, 16, 4, 4, gradhCorrection=1, XSPH=1,
                                                 compatibleEnergyEvolution=0) + (2, 2)
    c["crk_kh_crkq"] = _kh(gen, abi, 8, 8, 4, hydro=abi.HYDRO_CRKSPH, qType=abi.Q_CRKSPH_MONAGHAN_GINGOLD) + (2, 2)
    c["crk_sod"] = _sod(gen, abi, 16, 4, 4, hydro=abi.HYDRO_CRKSPH) + (2, 2)
    return c


def restart_fixture(exe, name, ns, cfg, nsteps, nmore):
    with tempfile.TemporaryDirectory() as td:
        write_input(os.path.join(td, "a.bin"), cfg, ns, nsteps)
        write_input(os.path.join(td, "b.bin"), cfg, ns, nmore)
        rst = os.path.join(td, "restart.txt")
        subprocess.check_call([exe, "--restart-dump", os.path.join(td, "a.bin"), rst], stdout=subprocess.DEVNULL)
        os.makedirs(os.path.join(td, "cont", "steps"))
        subprocess.check_call([exe, "--restart-load", os.path.join(td, "b.bin"), rst, os.path.join(td, "cont")],
                              stdout=subprocess.DEVNULL)
        with open(rst, "rb") as f:
            text = f.read()
        d = os.path.join(td, "cont", "steps")
        cont = {"cont/" + f[:-4]: np.fromfile(os.path.join(d, f), dtype="<f8")
                for f in sorted(os.listdir(d)) if f.endswith(".f64")}
    data = {"input/config": np.frombuffer(bytes(cfg), dtype=np.uint8), "input/nsteps": np.int64(nsteps),
            "input/nmore": np.int64(nmore), "input/position": ns.pos, "input/velocity": ns.vel,
            "input/mass": ns.mass, "input/mass density": ns.rho, "input/specific thermal energy": ns.eps,
            "input/H": ns.H, "restart": np.frombuffer(text, dtype=np.uint8)}
    data.update(cont)
    out = os.path.join(HERE, "reference_restart_%s.npz" % name)
    np.savez_compressed(out, **data)
    return out


def main(argv):
    build_ref = importlib.import_module("build_ref")
    ref_sph, ref_tables = build_ref.build()
    want = argv[1:]
    pkg = importlib.import_module("llnl-spheral_b200")
    for name, (ns, cfg) in idealh_cases(pkg).items():
        if want and "idealh_" + name not in want:
            continue
        print(idealh_fixture(ref_sph, name, ns, cfg))
    if not want or "tables" in want:
        with tempfile.TemporaryDirectory() as td:
            subprocess.check_call([ref_tables, td], stdout=subprocess.DEVNULL)
            data = {}
            for f in sorted(os.listdir(td)):
                if f.endswith(".f64"):
                    data[f[:-4]] = np.fromfile(os.path.join(td, f), dtype="<f8")
        out = os.path.join(HERE, "reference_tables.npz")
        np.savez_compressed(out, **data)
        print(out)
    pkg = importlib.import_module("llnl-spheral_b200")
    for name, (ns, cfg, nsteps) in cases(pkg).items():
        if want and name not in want:
            continue
        print(sph_fixture(ref_sph, name, ns, cfg, nsteps))
    for name, (ns, cfg, nsteps, nmore) in restart_cases(pkg).items():
        if want and "restart_" + name not in want:
            continue
        print(restart_fixture(ref_sph, name, ns, cfg, nsteps, nmore))


if __name__ == "__main__":
    main(sys.argv)
