// TEST INFRASTRUCTURE: stand-ins for reference entry points that the
// SPH/CRKSPH fluid path links but never calls at the configurations the
// checker runs (Voronoi meshes and volumes, hull and H volumes, surface
// detection, Peano-Hilbert redistribution).  Their sources need the polytope
// and qhull libraries, which are not installed.  Each stand-in aborts with a
// message if it is ever reached, except the empty Mesh's constructor,
// clear() and assignment, which the hydro objects call on a Mesh member they
// never fill.
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "Geometry/Dimension.hh"
#include "Mesh/Mesh.hh"
#include "Mesh/generateMesh.hh"
#include "Utilities/peanoHilbertOrderIndices.hh"
#include "Boundary/Boundary.hh"
#include "DataBase/DataBase.hh"
namespace {
[[noreturn]] void unreachable(const char* what) { std::fprintf(stderr, "reference stand-in reached: %s\n", what); std::abort(); }
}
namespace Spheral {
namespace MeshSpace {
template<> Mesh<Dim<3> >::Mesh() {}
template<> void Mesh<Dim<3> >::clear() {}
template<> Mesh<Dim<3> >& Mesh<Dim<3> >::operator=(const Mesh<Dim<3> >&) { return *this; }
template<> std::string Mesh<Dim<3> >::valid() const { unreachable("Mesh::valid"); }
template<> std::string Mesh<Dim<3> >::validDomainInfo(const Dim<3>::Vector&, const Dim<3>::Vector&, const bool) const { unreachable("Mesh::validDomainInfo"); }
template<> double Mesh<Dim<3> >::Zone::volume() const { unreachable("Mesh::Zone::volume"); }
typedef std::vector<const NodeSpace::NodeList<Dim<3> >*>::iterator NLI;
typedef std::vector<BoundarySpace::Boundary<Dim<3> >*>::const_iterator BI;
template<> void generateMesh<Dim<3>, NLI, BI>(const NLI, const NLI, const BI, const BI, const Dim<3>::Vector&, const Dim<3>::Vector&,
                                             const bool, const bool, const bool, const bool, const double, Mesh<Dim<3> >&,
                                             NodeSpace::NodeList<Dim<3> >&) { unreachable("generateMesh"); }
}
template<> FieldSpace::FieldList<Dim<3>, KeyTraits::Key> peanoHilbertOrderIndices<Dim<3> >(const DataBaseSpace::DataBase<Dim<3> >&) { unreachable("peanoHilbertOrderIndices"); }
}
#include "Geometry/GeomPolyhedron.hh"
#include "CRKSPH/computeVoronoiVolume.hh"
#include "CRKSPH/detectSurface.hh"
#include "CRKSPH/computeHVolumes.hh"
#include "CRKSPH/computeHullVolumes.hh"
namespace Spheral {
using namespace FieldSpace;
using namespace NeighborSpace;
typedef Dim<3> D3;
GeomPolyhedron::~GeomPolyhedron() {}
namespace CRKSPHSpace {
void computeVoronoiVolume(const FieldList<D3, D3::Vector>&, const FieldList<D3, D3::SymTensor>&, const FieldList<D3, D3::Scalar>&,
                          const FieldList<D3, D3::Vector>&, const ConnectivityMap<D3>&, const std::vector<D3::FacetedVolume>&,
                          const std::vector<std::vector<D3::FacetedVolume> >&, const FieldList<D3, D3::Scalar>&,
                          const FieldList<D3, int>&, FieldList<D3, int>&, FieldList<D3, D3::Scalar>&, FieldList<D3, D3::Vector>&,
                          FieldList<D3, std::vector<D3::Vector> >&, FieldList<D3, D3::FacetedVolume>&) { unreachable("computeVoronoiVolume"); }
template<> void detectSurface<D3>(const ConnectivityMap<D3>&, const FieldList<D3, D3::Scalar>&, const FieldList<D3, D3::Vector>&,
                                  const FieldList<D3, D3::Vector>&, const FieldList<D3, D3::SymTensor>&, const double, const double,
                                  const double, FieldList<D3, int>&) { unreachable("detectSurface"); }
}
template<> void computeHVolumes<D3>(const D3::Scalar, const FieldList<D3, D3::SymTensor>&, FieldList<D3, D3::Scalar>&) { unreachable("computeHVolumes"); }
template<> void computeHullVolumes<D3>(const ConnectivityMap<D3>&, const D3::Scalar, const FieldList<D3, D3::Vector>&,
                                       const FieldList<D3, D3::SymTensor>&, FieldList<D3, D3::Scalar>&) { unreachable("computeHullVolumes"); }
}
