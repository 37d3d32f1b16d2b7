// Host construction of TableKernel<Dim<3>> for the device tables.
//
// Follows the reference's construction so that the device lookups return
// the reference's numbers (compiled with -ffp-contract=off):
//   analytic kernels   src/Kernel/BSplineKernelInline.hh:27-101,
//                      src/Kernel/WendlandC4KernelInline.hh:27-103
//   table + fits       src/Kernel/TableKernel.cc:211-305, 472-506 (the 3x3
//                      fit matrix has the exact inverse
//                      [[1/2,-1,1/2],[-3/2,2,-1/2],[1,0,0]])
//   nPerh tables       src/Kernel/TableKernel.cc:64-93, 514-548
// The device table packs, per point i, (aK, bK, cK, aG, bG, cG).
#include <algorithm>
#include <cmath>
#include <vector>

namespace sphgpu {

namespace {

struct Analytic {
  int type;
  double norm, extent;
  explicit Analytic(int t) : type(t) {
    if (t == 0) { norm = 1.0/M_PI; extent = 2.0; }
    else        { norm = 495.0/(32.0*M_PI); extent = 1.0; }
  }
  double W(double eta) const {
    const double Hdet = 1.0;
    if (type == 0) {
      if (eta < 1.0) { double eta2 = eta*eta; return norm*Hdet*(1.0 - 1.5*eta2 + 0.75*eta2*eta); }
      if (eta < 2.0) { const double t = 2.0 - eta; return norm*Hdet*0.25*(t*t*t); }
      return 0.0;
    }
    double eta2 = eta*eta;
    return norm*Hdet*(std::pow(1.0 - eta, 6)*(1.0 + 6.0*eta + (35.0/3.0)*eta2))*(eta < 1.0);
  }
  double gW(double eta) const {
    const double Hdet = 1.0;
    if (type == 0) {
      if (eta < 1.0) return -norm*Hdet*(3.0 - 2.25*eta)*eta;
      if (eta < 2.0) { const double t = 2.0 - eta; return -norm*Hdet*0.75*(t*t); }
      return 0.0;
    }
    return norm*Hdet*((56.0/3.0)*std::pow(eta - 1.0, 5)*eta*(5.0*eta + 1.0))*(eta < 1.0);
  }
};

void fit(const std::vector<double>& t, int n, std::vector<double>& a, std::vector<double>& b,
         std::vector<double>& c) {
  static const double Ainv[3][3] = {{0.5, -1.0, 0.5}, {-1.5, 2.0, -0.5}, {1.0, -0.0, -0.0}};
  a.assign(n, 0.0); b.assign(n, 0.0); c.assign(n, 0.0);
  for (int i0 = 0; i0 < n - 2; ++i0) {
    const double B[3] = {t[i0], t[i0 + 1], t[i0 + 2]};
    double C[3];
    for (int r = 0; r < 3; ++r) {
      double s = Ainv[r][0]*B[0];
      s += Ainv[r][1]*B[1];
      s += Ainv[r][2]*B[2];
      C[r] = s;
    }
    a[i0 + 1] = C[2]; b[i0 + 1] = C[1]; c[i0 + 1] = C[0];
  }
}

bool fuzzyZero(double x) { return std::abs(x)/std::max(1.0, std::abs(x)) < 1.0e-15; }

}  // namespace

double table_kernel_value(const std::vector<double>& coef6, int n, double stepSize, double extent,
                          double eta, double Hdet) {
  if (!(eta < extent)) return 0.0;
  const double q = eta/stepSize;
  const int lb = std::min(n - 1, int(q));
  const int i0 = std::min(n - 3, lb);
  const int i1 = i0 + 1;
  const double x = q - i0;
  const double* c = coef6.data() + 6*size_t(i1);
  return Hdet*(c[0] + c[1]*x + c[2]*x*x);
}

static double table_grad_value(const std::vector<double>& coef6, int n, double stepSize, double extent,
                               double eta) {
  if (!(eta < extent)) return 0.0;
  const double q = eta/stepSize;
  const int lb = std::min(n - 1, int(q));
  const int i0 = std::min(n - 3, lb);
  const double x = q - i0;
  const double* c = coef6.data() + 6*size_t(i0 + 1);
  return 1.0*(c[3] + c[4]*x + c[5]*x*x);
}

void build_table_kernel(int kernelType, int numPoints, std::vector<double>& coef6, std::vector<double>& nperh,
                        std::vector<double>& wsum, double& stepSize, double& extent) {
  const Analytic k(kernelType);
  const int n = numPoints;
  extent = 1.0*k.extent;
  stepSize = extent/(n - 1);
  std::vector<double> kv(n), gv(n);
  const double correction = 1.0/(1.0*1.0*1.0);
  const double deta = stepSize/1.0;
  for (int i = 0; i < n; ++i) {
    kv[i] = correction*k.W(i*deta);
    gv[i] = correction*k.gW(i*deta);
  }
  std::vector<double> aK, bK, cK, aG, bG, cG;
  fit(kv, n, aK, bK, cK);
  fit(gv, n, aG, bG, cG);
  coef6.assign(6*size_t(n), 0.0);
  for (int i = 0; i < n; ++i) {
    double* c = coef6.data() + 6*size_t(i);
    c[0] = aK[i]; c[1] = bK[i]; c[2] = cK[i]; c[3] = aG[i]; c[4] = bG[i]; c[5] = cG[i];
  }
  // nPerh <-> Wsum tables (3-D lattice sum of |grad W|).
  const double minNperh = 0.25, maxNperh = 10.0;
  nperh.assign(n, 0.0);
  wsum.assign(n, 0.0);
  const double dnperh = (maxNperh - minNperh)/(n - 1);
  for (int i = 0; i != n; ++i) {
    const double np = minNperh + i*dnperh;
    const double d = 1.0/np;
    nperh[i] = np;
    double result = 0.0;
    double ez = 0.0;
    while (ez < extent) {
      double ey = 0.0;
      while (ey < extent) {
        double ex = 0.0;
        while (ex < extent) {
          const double m = std::sqrt(ex*ex + ey*ey + ez*ez);
          double dr = std::abs(table_grad_value(coef6, n, stepSize, extent, m));
          if (ex > 0.0 && !fuzzyZero(ex)) dr *= 2.0;
          if (ey > 0.0 && !fuzzyZero(ey)) dr *= 2.0;
          if (ez > 0.0 && !fuzzyZero(ez)) dr *= 2.0;
          if (fuzzyZero(m)) dr *= 0.0;
          result += dr;
          ex += d;
        }
        ey += d;
      }
      ez += d;
    }
    wsum[i] = (result < 0.0 ? -1.0 : 1.0)*std::pow(std::abs(result), 0.3333333333333333);
  }
}

}  // namespace sphgpu
