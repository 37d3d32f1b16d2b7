// TEST INFRASTRUCTURE: a checker built from the reference's own sources.
//
// Compiles, unmodified from the reference source tree, TableKernel
// (src/Kernel/TableKernel.cc), the BSpline and Wendland C4 kernels, the
// Dim<3> geometry headers, GeomPlane (src/Geometry/GeomPlane.cc) and
// mapPositionThroughPlanes, against the stand-ins in oracle/refshim for the
// uninstalled Eigen / boost headers.  It writes golden vectors (raw float64
// little-endian) into the directory given on the command line; the test
// fixture script tests/golden/make_golden.py turns them into .npz files.
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "Geometry/Dimension.hh"
#include "Geometry/GeomPlane.hh"
#include "Kernel/TableKernel.hh"
#include "Kernel/BSplineKernel.hh"
#include "Kernel/WendlandC4Kernel.hh"
#include "Boundary/mapPositionThroughPlanes.hh"
// template definitions instantiated in this translation unit
#include "Kernel/TableKernel.cc"
#include "Geometry/GeomPlane.cc"

using namespace Spheral;
using namespace Spheral::KernelSpace;
typedef Dim<3>::Vector Vector;
typedef Dim<3>::SymTensor SymTensor;

namespace {

uint64_t g_state = 0x20261203ULL;
double urand() {  // splitmix64 -> [0,1)
  uint64_t z = (g_state += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30))*0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27))*0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return (z >> 11)*(1.0/9007199254740992.0);
}

void dump(const std::string& dir, const std::string& name, const std::vector<double>& v) {
  const std::string path = dir + "/" + name + ".f64";
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) { std::perror(path.c_str()); std::exit(1); }
  std::fwrite(v.data(), sizeof(double), v.size(), f);
  std::fclose(f);
}

template<typename K>
void tables(const std::string& dir, const std::string& tag, const K& base, int numPoints) {
  const TableKernel<Dim<3> > W(base, numPoints);
  std::vector<double> eta, Wv, gWv;
  const double ext = W.kernelExtent();
  const int ns = 4001;
  for (int i = 0; i < ns; ++i) eta.push_back(ext*1.02*i/(ns - 1));   // crosses the support edge
  for (int i = 0; i < 2000; ++i) eta.push_back(ext*urand());
  for (double e : eta) {
    const std::pair<double, double> r = W.kernelAndGradValue(e, 1.0);
    Wv.push_back(r.first);
    gWv.push_back(r.second);
  }
  dump(dir, tag + "_eta", eta);
  dump(dir, tag + "_W", Wv);
  dump(dir, tag + "_gW", gWv);
  dump(dir, tag + "_nperh", W.nperhValues());
  dump(dir, tag + "_wsum", W.WsumValues());
  std::vector<double> ws, np;
  const std::vector<double>& wt = W.WsumValues();
  for (int i = 0; i < 1000; ++i) ws.push_back(wt.front()*0.5 + (wt.back()*1.2 - wt.front()*0.5)*urand());
  for (double x : ws) np.push_back(W.equivalentNodesPerSmoothingScale(x));
  dump(dir, tag + "_wsum_query", ws);
  dump(dir, tag + "_nperh_query", np);
  std::vector<double> an;
  for (double e : eta) { an.push_back(base.kernelValue(e, 1.0)); an.push_back(base.gradValue(e, 1.0)); }
  dump(dir, tag + "_analytic", an);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) { std::fprintf(stderr, "usage: %s outdir\n", argv[0]); return 2; }
  const std::string dir = argv[1];
  tables(dir, "bspline", BSplineKernel<Dim<3> >(), 1000);
  tables(dir, "wendlandc4", WendlandC4Kernel<Dim<3> >(), 1000);

  // SymTensor / Vector operations on random (positive definite) H and r.
  std::vector<double> Hin, rin, out;
  for (int s = 0; s < 512; ++s) {
    const bool iso = s < 128;
    const double h = 50.0 + 200.0*urand();
    double a[6];
    if (iso) { a[0] = h; a[1] = 0.0; a[2] = 0.0; a[3] = h; a[4] = 0.0; a[5] = h; }
    else {
      a[0] = h*(1.0 + urand()); a[3] = h*(1.0 + urand()); a[5] = h*(1.0 + urand());
      a[1] = 0.2*h*(urand() - 0.5); a[2] = 0.2*h*(urand() - 0.5); a[4] = 0.2*h*(urand() - 0.5);
    }
    const SymTensor H(a[0], a[1], a[2], a[1], a[3], a[4], a[2], a[4], a[5]);
    const Vector r(urand() - 0.5, urand() - 0.5, urand() - 0.5);
    for (int k = 0; k < 6; ++k) Hin.push_back(a[k]);
    rin.push_back(r.x()); rin.push_back(r.y()); rin.push_back(r.z());
    const Vector ev = H.eigenValues();
    out.push_back(ev.x()); out.push_back(ev.y()); out.push_back(ev.z());
    out.push_back(H.Determinant());
    const SymTensor Hi = H.Inverse();
    out.push_back(Hi.xx()); out.push_back(Hi.xy()); out.push_back(Hi.xz());
    out.push_back(Hi.yy()); out.push_back(Hi.yz()); out.push_back(Hi.zz());
    const Vector hr = H*r;
    out.push_back(hr.x()); out.push_back(hr.y()); out.push_back(hr.z());
    const Vector u = r.unitVector();
    out.push_back(u.x()); out.push_back(u.y()); out.push_back(u.z());
  }
  dump(dir, "geom_H", Hin);
  dump(dir, "geom_r", rin);
  dump(dir, "geom_out", out);

  // Periodic plane mapping of a box [0,1]x[0,0.125]x[0,0.125] (ghost images
  // through PlanarBoundary(enter, exit): mapPosition(pos, exit, enter)).
  const Vector xmin(0.0, 0.0, 0.0), xmax(1.0, 0.125, 0.125);
  std::vector<double> pin, pout;
  for (int s = 0; s < 256; ++s) {
    const Vector p(-0.05 + 1.1*urand(), -0.02 + 0.165*urand(), -0.02 + 0.165*urand());
    pin.push_back(p.x()); pin.push_back(p.y()); pin.push_back(p.z());
  }
  for (int axis = 0; axis < 3; ++axis) {
    Vector n0(0.0, 0.0, 0.0), n1(0.0, 0.0, 0.0);
    n0(axis) = 1.0; n1(axis) = -1.0;
    const GeomPlane<Dim<3> > plane1(xmin, n0), plane2(xmax, n1);
    for (int which = 0; which < 2; ++which) {
      const GeomPlane<Dim<3> >& enter = which == 0 ? plane1 : plane2;
      const GeomPlane<Dim<3> >& exit = which == 0 ? plane2 : plane1;
      for (int s = 0; s < 256; ++s) {
        const Vector p(pin[3*s], pin[3*s + 1], pin[3*s + 2]);
        const Vector g = mapPositionThroughPlanes(p, exit, enter);
        pout.push_back(g.x()); pout.push_back(g.y()); pout.push_back(g.z());
      }
    }
  }
  dump(dir, "map_in", pin);
  dump(dir, "map_out", pout);
  std::printf("ok\n");
  return 0;
}
