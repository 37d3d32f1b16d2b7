// TEST INFRASTRUCTURE -- part of the CPU oracle (see geom.hh header).
//
// TableKernel<Dim<3>> restated from the reference:
//   analytic kernels  src/Kernel/BSplineKernelInline.hh:27-101,
//                     src/Kernel/WendlandC4KernelInline.hh:27-103
//   construction      src/Kernel/TableKernel.cc:211-305 (hmult = 1)
//   parabolic fits    src/Kernel/TableKernel.cc:472-506 (Eigen 3x3 inverse of
//                     [[0,0,1],[1,1,1],[4,2,1]], exact in FP64)
//   nPerh tables      src/Kernel/TableKernel.cc:64-93 (3-D sumKernelValues),
//                     :514-548 (setNperhValues), :402-430
//                     (equivalentNodesPerSmoothingScale), bisectSearch
//                     src/Utilities/bisectSearch.hh
//   lookups           src/Kernel/TableKernelInline.hh:11-78,262-294
#ifndef ORACLE_TABLE_KERNEL_HH
#define ORACLE_TABLE_KERNEL_HH

#include <cmath>
#include <vector>
#include <utility>

#include "geom.hh"

namespace orc {

struct BaseKernel {
  int type;          // 0 BSpline, 1 WendlandC4
  double norm, extent;
  explicit BaseKernel(int t): type(t) {
    if (t == 0) { norm = 1.0/M_PI; extent = 2.0; }
    else        { norm = 495.0/(32.0*M_PI); extent = 1.0; }
  }
  double kernelValue(double eta, double Hdet) const {
    if (type == 0) {
      if (eta < 1.0) {
        double eta2 = eta*eta;
        return norm*Hdet*(1.0 - 1.5*eta2 + 0.75*eta2*eta);
      } else if (eta < 2.0) {
        const double t = 2.0 - eta;
        return norm*Hdet*0.25*(t*t*t);
      }
      return 0.0;
    }
    double eta2 = eta*eta;
    return norm*Hdet*(std::pow(1.0 - eta, 6)*(1.0 + 6.0*eta + (35.0/3.0)*eta2))*(eta < 1.0);
  }
  double gradValue(double eta, double Hdet) const {
    if (type == 0) {
      if (eta < 1.0) return -norm*Hdet*(3.0 - 2.25*eta)*eta;
      else if (eta < 2.0) { const double t = 2.0 - eta; return -norm*Hdet*0.75*(t*t); }
      return 0.0;
    }
    return norm*Hdet*((56.0/3.0)*std::pow(eta - 1.0, 5)*eta*(5.0*eta + 1.0))*(eta < 1.0);
  }
  double grad2Value(double eta, double Hdet) const {
    if (type == 0) {
      if (eta < 1.0) return -norm*Hdet*(3 - 4.5*eta);
      else if (eta < 2.0) return norm*Hdet*1.5*(2 - eta);
      return 0.0;
    }
    const double eta2 = eta*eta;
    return norm*Hdet*((56.0/3.0)*std::pow(eta - 1.0, 4)*(35.0*eta2 - 4.0*eta - 1.0))*(eta < 1.0);
  }
};

struct TableKernel {
  int n = 0;
  double extent = 0.0, stepSize = 0.0;
  double minNperh = 0.25, maxNperh = 10.0;
  std::vector<double> aK, bK, cK, aG, bG, cG, aG2, bG2, cG2, nperh, wsum;

  TableKernel() {}
  TableKernel(int kernelType, int numPoints) {
    const BaseKernel k(kernelType);
    const double hmult = 1.0;
    extent = hmult*k.extent;
    n = numPoints;
    stepSize = extent/(numPoints - 1);
    std::vector<double> kv(n), gv(n), g2v(n);
    const double correction = 1.0/(hmult*hmult*hmult);
    const double deta = stepSize/hmult;
    for (int i = 0; i < n; ++i) {
      kv[i] = correction*k.kernelValue(i*deta, 1.0);
      gv[i] = correction*k.gradValue(i*deta, 1.0);
      g2v[i] = correction*k.grad2Value(i*deta, 1.0);
    }
    setParabolicCoeffs(kv, aK, bK, cK);
    setParabolicCoeffs(gv, aG, bG, cG);
    setParabolicCoeffs(g2v, aG2, bG2, cG2);
    setNperhValues();
  }

  void setParabolicCoeffs(const std::vector<double>& t, std::vector<double>& a,
                          std::vector<double>& b, std::vector<double>& c) const {
    // Rows of inverse([[0,0,1],[1,1,1],[4,2,1]]), times B = (t0, t1, t2),
    // each row summed left to right.
    static const double Ainv[3][3] = {{0.5, -1.0, 0.5}, {-1.5, 2.0, -0.5}, {1.0, -0.0, -0.0}};
    a.assign(n, 0.0); b.assign(n, 0.0); c.assign(n, 0.0);
    for (int i0 = 0; i0 < n - 2; ++i0) {
      const int i1 = i0 + 1, i2 = i0 + 2;
      const double B0 = t[i0], B1 = t[i1], B2 = t[i2];
      double C[3];
      for (int r = 0; r < 3; ++r) {
        double s = Ainv[r][0]*B0;
        s += Ainv[r][1]*B1;
        s += Ainv[r][2]*B2;
        C[r] = s;
      }
      a[i1] = C[2]; b[i1] = C[1]; c[i1] = C[0];
    }
  }

  int lowerBound(double eta) const { return std::min(n - 1, int(eta/stepSize)); }

  double parabolicInterp(double eta, const std::vector<double>& a, const std::vector<double>& b,
                         const std::vector<double>& c) const {
    const int i0 = std::min(n - 3, lowerBound(eta));
    const int i1 = i0 + 1;
    const double x = eta/stepSize - i0;
    return a[i1] + b[i1]*x + c[i1]*x*x;
  }
  double kernelValue(double eta, double Hdet) const {
    return eta < extent ? Hdet*parabolicInterp(eta, aK, bK, cK) : 0.0;
  }
  double gradValue(double eta, double Hdet) const {
    return eta < extent ? Hdet*parabolicInterp(eta, aG, bG, cG) : 0.0;
  }
  double grad2Value(double eta, double Hdet) const {
    return eta < extent ? Hdet*parabolicInterp(eta, aG2, bG2, cG2) : 0.0;
  }
  std::pair<double, double> kernelAndGradValue(double eta, double Hdet) const {
    if (eta < extent) {
      const int i0 = std::min(n - 3, lowerBound(eta));
      const int i1 = i0 + 1;
      const double x = eta/stepSize - i0;
      return std::make_pair(Hdet*(aK[i1] + bK[i1]*x + cK[i1]*x*x),
                            Hdet*(aG[i1] + bG[i1]*x + cG[i1]*x*x));
    }
    return std::make_pair(0.0, 0.0);
  }

  double sumKernelValues(double deta) const {
    double result = 0.0;
    double etaz = 0.0;
    while (etaz < extent) {
      double etay = 0.0;
      while (etay < extent) {
        double etax = 0.0;
        while (etax < extent) {
          const V3 eta{etax, etay, etaz};
          double dresult = std::abs(gradValue(mag(eta), 1.0));
          if (distinctlyGreaterThan(etax, 0.0)) dresult *= 2.0;
          if (distinctlyGreaterThan(etay, 0.0)) dresult *= 2.0;
          if (distinctlyGreaterThan(etaz, 0.0)) dresult *= 2.0;
          if (fuzzyEqual(mag(eta), 0.0)) dresult *= 0.0;
          result += dresult;
          etax += deta;
        }
        etay += deta;
      }
      etaz += deta;
    }
    return CubeRootHalley2(result);
  }

  void setNperhValues() {
    wsum.assign(n, 0.0);
    nperh.assign(n, 0.0);
    const double dnperh = (maxNperh - minNperh)/(n - 1);
    for (int i = 0; i != n; ++i) {
      const double np = minNperh + i*dnperh;
      const double deta = 1.0/np;
      nperh[i] = np;
      wsum[i] = sumKernelValues(deta);
    }
  }

  static int bisectSearch(const std::vector<double>& t, double val) {
    const int nn = int(t.size());
    if (nn > 1) {
      const bool ascnd = (t[nn - 1] >= t[0]);
      int jl = -1, ju = nn;
      while (ju - jl > 1) {
        const int jm = (ju + jl)/2;
        if ((val >= t[jm]) == ascnd) jl = jm; else ju = jm;
      }
      return jl;
    } else if (nn == 1) {
      return val <= t[0] ? -1 : 0;
    }
    return -1;
  }

  double equivalentNodesPerSmoothingScale(double Wsum) const {
    const int lb = bisectSearch(wsum, Wsum);
    const int ub = lb + 1;
    if (lb == -1) return nperh[0];
    if (ub == n) return nperh[n - 1];
    return std::min(nperh[ub],
                    std::max(nperh[lb],
                             nperh[lb] +
                             (Wsum - wsum[lb])/
                             (wsum[ub] - wsum[lb])*
                             (nperh[ub] - nperh[lb])));
  }
};

}  // namespace orc

#endif
