"""TEST INFRASTRUCTURE: build the checkers that run the reference's own code.

Compiles, with g++ directly, the reference's own sources where they lie in
the reference tree (nothing is copied), against the stand-in headers in
oracle/refshim (a 3x3 Eigen subset and a few boost pieces; neither library is
installed here), into oracle/_ref/:

  ref_tables  TableKernel, BSpline / Wendland C4, Dim<3> geometry, GeomPlane
              and mapPositionThroughPlanes (oracle/refshim/ref_tables.cc)
  ref_sph_gpu ref_sph with the drop-in adapter
              llnl-spheral_b200/spheral/GpuSPHHydroBase.hh in place of
              SPHHydroBase (its evaluateDerivatives on the GPU through
              llnl-spheral_b200/_build/libsphgpu.so, found at run time by a
              relative rpath); built when that library exists
  ref_sph     the whole SPH / CRKSPH fluid path: FluidNodeList,
              NestedGridNeighbor, ConnectivityMap, PeriodicBoundary, DataBase,
              State and its update policies, SPHHydroBase, CRKSPHHydroBase, the
              CRKSPH moment / correction / volume / density functions,
              MonaghanGingoldViscosity, CRKSPHMonaghanGingoldViscosity,
              SPHSmoothingScale, GammaLawGas, GenericHydro, Integrator,
              CheapSynchronousRK2 and iterateIdealH (oracle/refshim/ref_sph.cc)

Every reference translation unit is compiled on its own, followed by one
hand-written explicit instantiation for Dim<3> (the reference generates those
lines with Python 2 scripts at build time; they are written out here
instead).  Flags: -O2 -ffp-contract=off -fno-fast-math, no OpenMP, as for the
oracle.  The reference's own build system (autoconf + make) is not run.

The reference tree is found through $SPHERAL_REFERENCE, else at the path this
development container mounts it.  The GPU box has no reference tree; the tests
there read the committed fixtures in tests/golden/ only.

    python oracle/build_ref.py [--if-present] [-j N]
"""
import argparse
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SHIM = os.path.join(HERE, "refshim")
INCLUDE = os.path.join(HERE, "..", "include")
PKG = os.path.join(HERE, "..", "llnl-spheral_b200")


def reference_src():
    root = os.environ.get("SPHERAL_REFERENCE") or "/root/reference"
    return os.path.join(root, "src")


D3 = "Spheral::Dim<3> "
USING = ("namespace Spheral { using namespace FieldSpace; using namespace NeighborSpace; "
         "using namespace KernelSpace; using namespace DataBaseSpace; using namespace NodeSpace;\n%s\n}")


def _classes(name, args):
    return USING % "\n".join("template class %s<%s>;" % (name, a) for a in args)


def _fl(t):
    return "FieldList<Dim<3>, Dim<3>::%s>" % t


_S, _V, _V3, _T, _ST = ("Dim<3>::Scalar", "Dim<3>::Vector", "Dim<3>::Vector3d", "Dim<3>::Tensor",
                        "Dim<3>::SymTensor")
_FIVE = ["Dim<3>, " + x for x in (_S, _V, _V3, _T, _ST)]
_SIX = _FIVE + ["Dim<3>, %s, %s" % (_ST, _S)]
_MOMENTS = ", ".join("const %s&" % _fl(t) for t in ("Scalar", "Vector", "SymTensor", "ThirdRankTensor",
                                                     "FourthRankTensor", "Vector", "Tensor", "ThirdRankTensor",
                                                     "FourthRankTensor", "FifthRankTensor", "SymTensor"))
_CORR_OUT = ", ".join("%s&" % _fl(t) for t in ("Scalar", "Vector", "Tensor", "Vector", "Tensor", "ThirdRankTensor"))

# (reference source, explicit instantiation that follows it)
UNITS = [
    ("Geometry/Dimension.cc", ""), ("Geometry/GeomVector.cc", ""), ("Geometry/Geom3Vector.cc", ""),
    ("Geometry/GeomTensor.cc", ""), ("Geometry/GeomSymmetricTensor.cc", ""),
    ("Geometry/GeomThirdRankTensor.cc", ""), ("Geometry/GeomFourthRankTensor.cc", ""),
    ("Geometry/GeomFifthRankTensor.cc", ""), ("Geometry/GeomPlane.cc", ""),
    ("Material/PhysicalConstants.cc", ""),
    ("Material/EquationOfState.cc", "template class Spheral::Material::EquationOfState<%s>;" % D3),
    ("Material/GammaLawGas.cc", "template class Spheral::Material::GammaLawGas<%s>;" % D3),
    ("Kernel/TableKernel.cc",
     '#include "Kernel/BSplineKernel.hh"\n#include "Kernel/WendlandC4Kernel.hh"\n'
     "namespace Spheral { namespace KernelSpace {\ntemplate class TableKernel<Dim<3> >;\n"
     "template TableKernel<Dim<3> >::TableKernel(const BSplineKernel<Dim<3> >&, const int, const double);\n"
     "template TableKernel<Dim<3> >::TableKernel(const WendlandC4Kernel<Dim<3> >&, const int, const double);\n} }"),
    ("NodeList/NodeList.cc", "template class Spheral::NodeSpace::NodeList<%s>;" % D3),
    ("NodeList/FluidNodeList.cc", "template class Spheral::NodeSpace::FluidNodeList<%s>;" % D3),
    ("NodeList/SmoothingScaleBase.cc", "template class Spheral::NodeSpace::SmoothingScaleBase<%s>;" % D3),
    ("NodeList/SPHSmoothingScale.cc", "template class Spheral::NodeSpace::SPHSmoothingScale<%s>;" % D3),
    ("NodeList/NodeListRegistrar.cc",
     "template<typename Dimension> Spheral::NodeListRegistrar<Dimension>* "
     "Spheral::NodeListRegistrar<Dimension>::mInstancePtr = 0;\n"
     "template class Spheral::NodeListRegistrar<%s>;" % D3),
    ("Neighbor/Neighbor.cc", "template class Spheral::NeighborSpace::Neighbor<%s>;" % D3),
    ("Neighbor/NestedGridNeighbor.cc",
     "namespace Spheral { namespace NeighborSpace {\n"
     "template<> const double NestedGridNeighbor<Dim<3> >::ln2inverse = 1.0/log(2.0);\n"
     "template<> const int NestedGridNeighbor<Dim<3> >::mEndOfLinkList = -1;\n"
     "template<> const int NestedGridNeighbor<Dim<3> >::mGridNormalMagnitude = 1024;\n"
     "template class NestedGridNeighbor<Dim<3> >;\n} }"),
    ("Neighbor/ConnectivityMap.cc", "template class Spheral::NeighborSpace::ConnectivityMap<%s>;" % D3),
    ("Neighbor/GridCellIndex.cc",
     "#define INDEXMAX 1048576 - 1\n#define INDEXMIN -INDEXMAX - 1\n"
     "namespace Spheral { namespace NeighborSpace {\n"
     "template<> const int GridCellIndex<Dim<3> >::mIndexMax = INDEXMAX;\n"
     "template<> const int GridCellIndex<Dim<3> >::mIndexMin = INDEXMIN;\n} }"),
    ("Neighbor/GridCellPlane.cc", "template class Spheral::NeighborSpace::GridCellPlane<%s>;" % D3),
    ("DataBase/DataBase.cc", "template class Spheral::DataBaseSpace::DataBase<%s>;" % D3),
    ("DataBase/StateBase.cc", "template class Spheral::StateBase<%s>;" % D3),
    ("DataBase/State.cc", "template class Spheral::State<%s>;" % D3),
    ("DataBase/StateDerivatives.cc", "template class Spheral::StateDerivatives<%s>;" % D3),
    ("DataBase/CompositeFieldListPolicy.cc", _classes("CompositeFieldListPolicy", _FIVE)),
    ("DataBase/IncrementFieldList.cc", _classes("IncrementFieldList", _FIVE)),
    ("DataBase/IncrementBoundedState.cc", _classes("IncrementBoundedState", _SIX)),
    ("DataBase/ReplaceBoundedState.cc", _classes("ReplaceBoundedState", _SIX)),
    ("DataBase/IncrementBoundedFieldList.cc", _classes("IncrementBoundedFieldList", _SIX)),
    ("DataBase/ReplaceBoundedFieldList.cc", _classes("ReplaceBoundedFieldList", _SIX)),
    ("DataBase/ReplaceFieldList.cc", _classes("ReplaceFieldList", _FIVE)),
    ("DataBase/IncrementState.cc", _classes("IncrementState", _FIVE)),
    ("DataBase/ReplaceState.cc", _classes("ReplaceState", _FIVE)),
    ("DataBase/CopyState.cc", _classes("CopyState", _FIVE)),
    ("DataBase/CopyFieldList.cc", _classes("CopyFieldList", _FIVE)),
    ("Field/AllNodeIterator.cc", _classes("AllNodeIterator", ["Dim<3>"])),
    ("Field/InternalNodeIterator.cc", _classes("InternalNodeIterator", ["Dim<3>"])),
    ("Field/GhostNodeIterator.cc", _classes("GhostNodeIterator", ["Dim<3>"])),
    ("Field/MasterNodeIterator.cc", _classes("MasterNodeIterator", ["Dim<3>"])),
    ("Field/CoarseNodeIterator.cc", _classes("CoarseNodeIterator", ["Dim<3>"])),
    ("Field/RefineNodeIterator.cc", _classes("RefineNodeIterator", ["Dim<3>"])),
    ("Field/NodeIteratorBase.cc", _classes("NodeIteratorBase", ["Dim<3>"])),
    ("Boundary/Boundary.cc", "template class Spheral::BoundarySpace::Boundary<%s>;" % D3),
    ("Boundary/PlanarBoundary.cc", "template class Spheral::BoundarySpace::PlanarBoundary<%s>;" % D3),
    ("Boundary/PeriodicBoundary.cc", "template class Spheral::BoundarySpace::PeriodicBoundary<%s>;" % D3),
    ("Boundary/CRKSPHVoidBoundary.cc", "template class Spheral::BoundarySpace::CRKSPHVoidBoundary<%s>;" % D3),
    ("ArtificialViscosity/ArtificialViscosity.cc",
     "template class Spheral::ArtificialViscositySpace::ArtificialViscosity<%s>;" % D3),
    ("ArtificialViscosity/MonaghanGingoldViscosity.cc",
     "template class Spheral::ArtificialViscositySpace::MonaghanGingoldViscosity<%s>;" % D3),
    ("ArtificialViscosity/CRKSPHMonaghanGingoldViscosity.cc",
     "template class Spheral::ArtificialViscositySpace::CRKSPHMonaghanGingoldViscosity<%s>;" % D3),
    ("Hydro/HydroFieldNames.cc", ""),
    ("Strength/SolidFieldNames.cc", ""),
] + [("Hydro/%s.cc" % p, _classes(p, ["Dim<3>"]))
     for p in ("PressurePolicy", "SoundSpeedPolicy", "SpecificFromTotalThermalEnergyPolicy",
               "SpecificThermalEnergyPolicy", "PositionPolicy", "VolumePolicy", "VoronoiMassDensityPolicy",
               "SumVoronoiMassDensityPolicy", "EntropyPolicy")] + [
    ("Mesh/MeshPolicy.cc", _classes("MeshPolicy", ["Dim<3>"])),
    ("SPH/SPHHydroBase.cc", "template class Spheral::SPHSpace::SPHHydroBase<%s>;" % D3),
    ("SPH/computeSPHSumMassDensity.cc", USING % (
        "namespace SPHSpace { template void computeSPHSumMassDensity(const ConnectivityMap<Dim<3> >&, "
        "const TableKernel<Dim<3> >&, const bool, const %s&, const %s&, const %s&, %s&); }"
        % (_fl("Vector"), _fl("Scalar"), _fl("SymTensor"), _fl("Scalar")))),
    ("SPH/correctSPHSumMassDensity.cc", USING % (
        "namespace SPHSpace { template void correctSPHSumMassDensity(const ConnectivityMap<Dim<3> >&, "
        "const TableKernel<Dim<3> >&, const bool, const %s&, const %s&, const %s&, %s&); }"
        % (_fl("Vector"), _fl("Scalar"), _fl("SymTensor"), _fl("Scalar")))),
    ("SPH/computeSPHOmegaGradhCorrection.cc", USING % (
        "namespace SPHSpace { template void computeSPHOmegaGradhCorrection(const ConnectivityMap<Dim<3> >&, "
        "const TableKernel<Dim<3> >&, const %s&, const %s&, %s&); }"
        % (_fl("Vector"), _fl("SymTensor"), _fl("Scalar")))),
    ("SPH/computeSumVoronoiCellMassDensity.cc", USING % (
        "namespace SPHSpace { template void computeSumVoronoiCellMassDensity(const ConnectivityMap<Dim<3> >&, "
        "const TableKernel<Dim<3> >&, const %s&, const %s&, const %s&, const %s&, %s&); }"
        % (_fl("Vector"), _fl("Scalar"), _fl("Scalar"), _fl("SymTensor"), _fl("Scalar")))),
    ("CRKSPH/CRKSPHHydroBase.cc", "template class Spheral::CRKSPHSpace::CRKSPHHydroBase<%s>;" % D3),
    ("CRKSPH/computeCRKSPHMoments.cc", USING % (
        "namespace CRKSPHSpace { template void computeCRKSPHMoments(const ConnectivityMap<Dim<3> >&, "
        "const TableKernel<Dim<3> >&, const %s&, const %s&, const %s&, const CRKOrder, const NodeCoupling&, %s); }"
        % (_fl("Scalar"), _fl("Vector"), _fl("SymTensor"),
           ", ".join("%s&" % _fl(t) for t in ("Scalar", "Vector", "SymTensor", "ThirdRankTensor", "FourthRankTensor",
                                             "Vector", "Tensor", "ThirdRankTensor", "FourthRankTensor",
                                             "FifthRankTensor"))))),
    ("CRKSPH/computeCRKSPHCorrections.cc", USING % (
        "namespace CRKSPHSpace {\n"
        "template void computeCRKSPHCorrections(%s, const CRKOrder, %s);\n"
        "template void computeZerothCRKSPHCorrections(const %s&, const %s&, %s&, %s&);\n"
        "template void computeLinearCRKSPHCorrections(const %s&, const %s&, const %s&, const %s&, const %s&, "
        "const %s&, const %s&, %s&, %s&, %s&, %s&);\n"
        "template void computeQuadraticCRKSPHCorrections(%s, %s);\n}"
        % (_MOMENTS, _CORR_OUT, _fl("Scalar"), _fl("Vector"), _fl("Scalar"), _fl("Vector"),
           _fl("Scalar"), _fl("Vector"), _fl("SymTensor"), _fl("Vector"), _fl("Tensor"), _fl("ThirdRankTensor"),
           _fl("SymTensor"), _fl("Scalar"), _fl("Vector"), _fl("Vector"), _fl("Tensor"), _MOMENTS, _CORR_OUT))),
    ("CRKSPH/computeCRKSPHSumVolume.cc", USING % (
        "namespace CRKSPHSpace { template void computeCRKSPHSumVolume(const ConnectivityMap<Dim<3> >&, "
        "const TableKernel<Dim<3> >&, const %s&, const %s&, const %s&, %s&); }"
        % (_fl("Vector"), _fl("Scalar"), _fl("SymTensor"), _fl("Scalar")))),
    ("CRKSPH/computeCRKSPHSumMassDensity.cc", USING % (
        "namespace CRKSPHSpace { template void computeCRKSPHSumMassDensity(const ConnectivityMap<Dim<3> >&, "
        "const TableKernel<Dim<3> >&, const %s&, const %s&, const %s&, const %s&, const FieldList<Dim<3>, int>&, "
        "%s&); }" % (_fl("Vector"), _fl("Scalar"), _fl("Scalar"), _fl("SymTensor"), _fl("Scalar")))),
    ("CRKSPH/ContinuityVolumePolicy.cc", "template class Spheral::ContinuityVolumePolicy<%s>;" % D3),
    ("Physics/Physics.cc", "template class Spheral::PhysicsSpace::Physics<%s>;" % D3),
    ("Physics/GenericHydro.cc", "template class Spheral::PhysicsSpace::GenericHydro<%s>;" % D3),
    ("Integrator/Integrator.cc", "template class Spheral::IntegratorSpace::Integrator<%s>;" % D3),
    ("Integrator/CheapSynchronousRK2.cc", "template class Spheral::IntegratorSpace::CheapSynchronousRK2<%s>;" % D3),
    ("Utilities/DBC.cc", ""), ("Utilities/KeyTraits.cc", ""), ("Utilities/Process.cc", ""),
    ("Utilities/PeanoHilbertTransform.cc", ""),
    ("Utilities/globalBoundingVolumes.cc", USING % (
        "template void globalBoundingBox(const Field<Dim<3>, Dim<3>::Vector>&, Dim<3>::Vector&, Dim<3>::Vector&, "
        "const bool);\ntemplate void globalBoundingBox(const %s&, Dim<3>::Vector&, Dim<3>::Vector&, const bool);"
        % _fl("Vector"))),
    ("Utilities/mortonOrderIndices.cc", USING % (
        "template FieldList<Dim<3>, KeyTraits::Key> mortonOrderIndices<Dim<3> >(const %s&);\n"
        "template FieldList<Dim<3>, KeyTraits::Key> mortonOrderIndices<Dim<3> >(const DataBase<Dim<3> >&);\n"
        "template FieldList<Dim<3>, KeyTraits::Key> mortonOrderIndices<Dim<3> >(const DataBase<Dim<3> >&, "
        "const FieldList<Dim<3>, int>&);" % _fl("Vector"))),
    ("Utilities/iterateIdealH.cc", USING % (
        "template void iterateIdealH<Dim<3> >(DataBase<Dim<3> >&, const std::vector<BoundarySpace::Boundary<Dim<3> >*>&, "
        "const TableKernel<Dim<3> >&, const SmoothingScaleBase<Dim<3> >&, const int, const double, const double, "
        "const bool, const bool);")),
    ("DataOutput/RestartRegistrar.cc", ""),
    ("FileIO/FileIO.cc", ""),
    ("FileIO/FlatFileIO.cc", ""),
]

TABLE_UNITS = ["Geometry/Dimension.cc", "Geometry/GeomVector.cc", "Geometry/GeomTensor.cc",
               "Geometry/GeomSymmetricTensor.cc"]


def flags(ref):
    return ["-std=c++11", "-O2", "-ffp-contract=off", "-fno-fast-math", "-w", "-DSPHERAL3D", "-DCXXONLY",
            "-I" + SHIM, "-I" + ref, "-I" + INCLUDE]


def _compile(args):
    cxx, cflags, tu, obj, deps = args
    if os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps):
        return tu, 0, ""
    r = subprocess.run([cxx] + cflags + ["-c", tu, "-o", obj], capture_output=True, text=True)
    return tu, r.returncode, r.stderr


def _shim_files():
    out = []
    for d, _, fs in os.walk(SHIM):
        out += [os.path.join(d, f) for f in fs]
    return out


def build(jobs=None, quiet=True):
    ref = reference_src()
    if not os.path.isdir(ref):
        raise FileNotFoundError("reference source tree not found (set SPHERAL_REFERENCE)")
    cxx = os.environ.get("CXX", "g++")
    cflags = flags(ref)
    objdir = os.path.join(OUT, "obj")
    os.makedirs(objdir, exist_ok=True)
    shim = _shim_files() + [os.path.abspath(__file__), os.path.join(INCLUDE, "sphgpu.h")]
    tasks = []
    for src, inst in UNITS:
        name = src.replace("/", "_").replace(".", "_")
        tu = os.path.join(objdir, name + ".cc")
        text = '#include "%s"\n%s\n' % (src, inst)
        if not os.path.exists(tu) or open(tu).read() != text:
            with open(tu, "w") as f:
                f.write(text)
        tasks.append((cxx, cflags, tu, tu[:-3] + ".o", [tu, os.path.join(ref, src)] + shim))
    for drv in ("ref_stubs.cc", "ref_sph.cc", "ref_tables.cc"):
        tu = os.path.join(SHIM, drv)
        tasks.append((cxx, cflags, tu, os.path.join(objdir, drv[:-3] + ".o"), [tu] + shim))
    failed = []
    with concurrent.futures.ThreadPoolExecutor(jobs or os.cpu_count() or 4) as ex:
        for tu, rc, err in ex.map(_compile, tasks):
            if rc:
                failed.append(tu)
                sys.stderr.write("compile failed: %s\n%s\n" % (tu, err[-4000:]))
    if failed:
        raise RuntimeError("reference checker build failed (%d units)" % len(failed))
    unit_objs = [t[3] for t in tasks[:len(UNITS)]]
    links = {
        "ref_sph": unit_objs + [os.path.join(objdir, "ref_stubs.o"), os.path.join(objdir, "ref_sph.o")],
        "ref_tables": [os.path.join(objdir, u.replace("/", "_").replace(".", "_") + ".o") for u in TABLE_UNITS]
                      + [os.path.join(objdir, "ref_tables.o")],
    }
    for exe, objs in links.items():
        path = os.path.join(OUT, exe)
        if os.path.exists(path) and all(os.path.getmtime(path) >= os.path.getmtime(o) for o in objs):
            continue
        subprocess.check_call([cxx, "-o", path] + objs)
    # the same driver with the GPU adapter, linked against the CUDA library
    lib = os.path.join(PKG, "_build", "libsphgpu.so")
    if os.path.exists(lib):
        tu = os.path.join(SHIM, "ref_sph.cc")
        obj = os.path.join(objdir, "ref_sph_gpu.o")
        adapter = os.path.join(PKG, "spheral", "GpuSPHHydroBase.hh")
        _, rc, err = _compile((cxx, cflags + ["-DREF_SPH_GPU", "-I" + os.path.join(PKG, "spheral")], tu, obj,
                               [tu, adapter] + shim))
        if rc:
            raise RuntimeError("ref_sph_gpu build failed:\n" + err[-4000:])
        path = os.path.join(OUT, "ref_sph_gpu")
        objs = unit_objs + [os.path.join(objdir, "ref_stubs.o"), obj]
        if not (os.path.exists(path) and all(os.path.getmtime(path) >= os.path.getmtime(o) for o in objs + [lib])):
            rpath = os.path.relpath(os.path.dirname(lib), OUT)
            subprocess.check_call([cxx, "-o", path] + objs + ["-L" + os.path.dirname(lib), "-lsphgpu",
                                                              "-Wl,-rpath,$ORIGIN/" + rpath])
    if not quiet:
        print(os.path.join(OUT, "ref_sph"))
    return os.path.join(OUT, "ref_sph"), os.path.join(OUT, "ref_tables")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--if-present", action="store_true", help="do nothing when the reference tree is absent")
    ap.add_argument("-j", type=int, default=None)
    a = ap.parse_args()
    if a.if_present and not os.path.isdir(reference_src()):
        return 0
    build(a.j, quiet=False)
    return 0


if __name__ == "__main__":
    sys.exit(main())
