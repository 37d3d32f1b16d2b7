// TEST INFRASTRUCTURE -- part of the CPU oracle.  Only tests/, the smoke check
// and bench.py's cpu_baseline leg may build, load or call anything in oracle/.
//
// Dim<3> geometry primitives restated with the reference's exact FP64
// expression order (build with -ffp-contract=off so no FMA is formed):
//   GeomVector<3>          src/Geometry/GeomVectorInline_default.hh:395-575,795-1045
//   GeomSymmetricTensor<3> src/Geometry/GeomSymmetricTensorInline_default.hh:895-955,1546-1661,2083-2109
//   GeomTensor<3>          src/Geometry/GeomTensorInline_default.hh:735-745,931-937,1327-1340,1817-1895,1918-1958
//   GeomPlane<3>           src/Geometry/GeomPlane.cc:41-46,218-259,308-313; src/Utilities/pointDistances.hh:53-57
//   FastMath / safeInv     src/Utilities/FastMath.hh:148-156,211-214; src/Utilities/safeInv.hh
#ifndef ORACLE_GEOM_HH
#define ORACLE_GEOM_HH

#include <algorithm>
#include <cmath>

namespace orc {

inline double sgn(const double x) { return x < 0.0 ? -1.0 : 1.0; }
inline bool fuzzyEqual(double lhs, double rhs, double fuzz = 1.0e-15) {
  return std::abs(lhs - rhs)/std::max(1.0, std::abs(lhs) + std::abs(rhs)) < fuzz;
}
inline bool distinctlyGreaterThan(double lhs, double rhs, double fuzz = 1.0e-15) {
  return lhs > rhs && !fuzzyEqual(lhs, rhs, fuzz);
}
inline double safeInv(double x, double fuzz = 1.0e-30) { return x/(x*x + fuzz); }
inline double safeInvVar(double x, double fuzz = 1.0e-30) { return sgn(x)/std::max(fuzz, std::abs(x)); }
// FastMath::CubeRootHalley2 under gcc (non-Intel branch).
inline double CubeRootHalley2(double d) { return sgn(d)*std::pow(std::abs(d), 0.3333333333333333); }
inline double pow4(double x) { return x*x*x*x; }

struct V3 {
  double x, y, z;
};
inline V3 vadd(const V3& a, const V3& b) { V3 r = a; r.x += b.x; r.y += b.y; r.z += b.z; return r; }
inline V3 vsub(const V3& a, const V3& b) { V3 r = a; r.x -= b.x; r.y -= b.y; r.z -= b.z; return r; }
inline V3 vneg(const V3& a) { return V3{-a.x, -a.y, -a.z}; }
// Vector*double and double*Vector (GeomVector::operator*=)
inline V3 vmul(const V3& a, double s) { V3 r = a; r.x *= s; r.y *= s; r.z *= s; return r; }
// Vector/double multiplies by the reciprocal (GeomVector<3>::operator/=)
inline V3 vdiv(const V3& a, double s) { const double inv = 1.0/s; return vmul(a, inv); }
inline double dot(const V3& a, const V3& b) { return a.x*b.x + a.y*b.y + a.z*b.z; }
inline double mag2(const V3& a) { return a.x*a.x + a.y*a.y + a.z*a.z; }
inline double mag(const V3& a) { return std::sqrt(a.x*a.x + a.y*a.y + a.z*a.z); }
inline V3 unitVector(const V3& a) {
  const double m = mag(a);
  return m > 1.0e-50 ? vdiv(a, m) : V3{1.0, 0.0, 0.0};
}
inline double maxAbsElement(const V3& a) { return std::max(std::abs(a.x), std::max(std::abs(a.y), std::abs(a.z))); }
inline double minElement(const V3& a) { return std::min(a.x, std::min(a.y, a.z)); }
inline double maxElement(const V3& a) { return std::max(a.x, std::max(a.y, a.z)); }

struct Sym {
  double xx, xy, xz, yy, yz, zz;
};
inline V3 sdot(const Sym& s, const V3& r) {
  return V3{s.xx*r.x + s.xy*r.y + s.xz*r.z,
            s.xy*r.x + s.yy*r.y + s.yz*r.z,
            s.xz*r.x + s.yz*r.y + s.zz*r.z};
}
inline double sdet(const Sym& s) {
  return (s.xx*s.yy*s.zz +
          s.xy*s.yz*s.xz +
          s.xz*s.xy*s.yz -
          s.xx*s.yz*s.yz -
          s.xy*s.xy*s.zz -
          s.xz*s.yy*s.xz);
}
inline Sym smul(const Sym& s, double v) {
  Sym r = s; r.xx *= v; r.xy *= v; r.xz *= v; r.yy *= v; r.yz *= v; r.zz *= v; return r;
}
inline Sym sdiv(const Sym& s, double v) { const double inv = 1.0/v; return smul(s, inv); }
inline Sym sadd(const Sym& a, const Sym& b) {
  Sym r = a; r.xx += b.xx; r.xy += b.xy; r.xz += b.xz; r.yy += b.yy; r.yz += b.yz; r.zz += b.zz; return r;
}
inline Sym sneg(const Sym& a) { return Sym{-a.xx, -a.xy, -a.xz, -a.yy, -a.yz, -a.zz}; }
inline Sym sinverse(const Sym& s) {
  const Sym c{s.yy*s.zz - s.yz*s.yz,
              s.yz*s.xz - s.xy*s.zz,
              s.xy*s.yz - s.yy*s.xz,
              s.xx*s.zz - s.xz*s.xz,
              s.xy*s.xz - s.xx*s.yz,
              s.xx*s.yy - s.xy*s.xy};
  return sdiv(c, sdet(s));
}
inline double smaxAbsElement(const Sym& s) {
  return std::max(std::abs(s.xx), std::max(std::abs(s.xy), std::max(std::abs(s.xz),
         std::max(std::abs(s.yy), std::max(std::abs(s.yz), std::abs(s.zz))))));
}
// Vector::selfdyad (src/Geometry/GeomVectorInline_default.hh:898-909)
inline Sym selfdyad(const V3& a) {
  const double A = a.x*a.x, B = a.x*a.y, C = a.x*a.z, D = a.y*a.y, E = a.y*a.z, F = a.z*a.z;
  return Sym{A, B, C, D, E, F};
}
// Analytic eigenvalues (src/Geometry/GeomSymmetricTensorInline_default.hh:2083-2109).
inline V3 eigenValues(const Sym& s) {
  static const double onethird = 1.0/3.0;
  static const double sqrt3 = std::sqrt(3.0);
  const double fscale = std::max(10.0*2.220446049250313e-16, smaxAbsElement(s));
  const double fscalei = 1.0/fscale;
  const double a00 = s.xx*fscalei, a01 = s.xy*fscalei, a02 = s.xz*fscalei;
  const double a11 = s.yy*fscalei, a12 = s.yz*fscalei, a22 = s.zz*fscalei;
  const double c0 = a00*a11*a22 + 2.0*a01*a02*a12 - a00*a12*a12 - a11*a02*a02 - a22*a01*a01;
  const double c1 = a00*a11 - a01*a01 + a00*a22 - a02*a02 + a11*a22 - a12*a12;
  const double c2 = a00 + a11 + a22;
  const double c2Div3 = c2*onethird;
  const double aDiv3 = std::min(0.0, onethird*(c1 - c2*c2Div3));
  const double mbDiv2 = 0.5*(c0 + c2Div3*(2.0*c2Div3*c2Div3 - c1));
  const double q = std::min(0.0, mbDiv2*mbDiv2 + aDiv3*aDiv3*aDiv3);
  const double m = std::sqrt(-aDiv3);
  const double angle = std::atan2(std::sqrt(-q), mbDiv2)*onethird;
  const double cs = std::cos(angle);
  const double sn = std::sin(angle);
  return V3{fscale*(c2Div3 + 2.0*m*cs),
            fscale*(c2Div3 - m*(cs + sqrt3*sn)),
            fscale*(c2Div3 - m*(cs - sqrt3*sn))};
}

struct T9 {
  double xx, xy, xz, yx, yy, yz, zx, zy, zz;
};
// GeomSymmetricTensor<3>::eigenVectors (src/Geometry/GeomSymmetricTensor_default.cc:36-95):
// scaled by the largest element, elements below 1e-20 zeroed, the 3x3
// eigenproblem solved, eigenvalues scaled back, eigenvector columns
// normalised.  The reference passes the solve to Eigen's
// SelfAdjointEigenSolver, which is not installed here; the solve restated is
// the cyclic Jacobi solver the reference checker links in its place
// (oracle/refshim/Eigen/Dense): rotations (0,1), (0,2), (1,2) per sweep until
// the off-diagonal mass is below 1e-32 of the diagonal, eigenvalues ascending.
struct Eig3 {
  V3 values;
  T9 vectors;   // column c: the eigenvector of values[c]
};
inline Eig3 symEigenVectors(const Sym& s) {
  const double fscale = std::max(10.0*2.220446049250313e-16, smaxAbsElement(s));
  const double fscalei = 1.0/fscale;
  const double e[6] = {s.xx*fscalei, s.xy*fscalei, s.xz*fscalei, s.yy*fscalei, s.yz*fscalei, s.zz*fscalei};
  double d[6];
  for (int k = 0; k < 6; ++k) d[k] = std::abs(e[k]) < 1.0e-20 ? 0.0 : e[k];
  double A[3][3] = {{d[0], d[1], d[2]}, {d[1], d[3], d[4]}, {d[2], d[4], d[5]}};
  double V[3][3] = {{1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
  for (int sweep = 0; sweep < 64; ++sweep) {
    const double off = A[0][1]*A[0][1] + A[0][2]*A[0][2] + A[1][2]*A[1][2];
    const double diag = A[0][0]*A[0][0] + A[1][1]*A[1][1] + A[2][2]*A[2][2];
    if (off <= 1e-32*diag || off == 0.0) break;
    for (int p = 0; p < 2; ++p) for (int q = p + 1; q < 3; ++q) {
      if (A[p][q] == 0.0) continue;
      const double theta = (A[q][q] - A[p][p])/(2.0*A[p][q]);
      const double t = (theta >= 0.0 ? 1.0 : -1.0)/(std::abs(theta) + std::sqrt(theta*theta + 1.0));
      const double c = 1.0/std::sqrt(t*t + 1.0), sn = t*c;
      for (int k = 0; k < 3; ++k) {
        const double akp = A[k][p], akq = A[k][q];
        A[k][p] = c*akp - sn*akq; A[k][q] = sn*akp + c*akq;
      }
      for (int k = 0; k < 3; ++k) {
        const double apk = A[p][k], aqk = A[q][k];
        A[p][k] = c*apk - sn*aqk; A[q][k] = sn*apk + c*aqk;
      }
      for (int k = 0; k < 3; ++k) {
        const double vkp = V[k][p], vkq = V[k][q];
        V[k][p] = c*vkp - sn*vkq; V[k][q] = sn*vkp + c*vkq;
      }
    }
  }
  int order[3] = {0, 1, 2};
  for (int i = 0; i < 3; ++i) for (int j = i + 1; j < 3; ++j)
    if (A[order[j]][order[j]] < A[order[i]][order[i]]) std::swap(order[i], order[j]);
  double B[3][3];
  for (int c = 0; c < 3; ++c) for (int r = 0; r < 3; ++r) B[r][c] = V[r][order[c]];
  Eig3 out;
  out.values = V3{A[order[0]][order[0]]*fscale, A[order[1]][order[1]]*fscale, A[order[2]][order[2]]*fscale};
  const double x1 = 1.0/std::sqrt(B[0][0]*B[0][0] + B[1][0]*B[1][0] + B[2][0]*B[2][0]);
  const double x2 = 1.0/std::sqrt(B[0][1]*B[0][1] + B[1][1]*B[1][1] + B[2][1]*B[2][1]);
  const double x3 = 1.0/std::sqrt(B[0][2]*B[0][2] + B[1][2]*B[1][2] + B[2][2]*B[2][2]);
  out.vectors = T9{B[0][0]*x1, B[0][1]*x2, B[0][2]*x3,
                   B[1][0]*x1, B[1][1]*x2, B[1][2]*x3,
                   B[2][0]*x1, B[2][1]*x2, B[2][2]*x3};
  return out;
}
// GeomSymmetricTensor<3>::rotationalTransform (src/Geometry/GeomSymmetricTensorInline_default.hh:1981-2014)
inline Sym rotationalTransform(const Sym& a, const T9& R) {
  const double A0 = a.xx, A1 = a.xy, A2 = a.xz, A3 = a.yy, A4 = a.yz, A5 = a.zz;
  const double R0 = R.xx, R1 = R.xy, R2 = R.xz, R3 = R.yx, R4 = R.yy, R5 = R.yz, R6 = R.zx, R7 = R.zy, R8 = R.zz;
  const double T0 = A0*R0 + A1*R1 + A2*R2;
  const double T1 = A0*R3 + A1*R4 + A2*R5;
  const double T2 = A1*R0 + A3*R1 + A4*R2;
  const double T3 = A1*R3 + A3*R4 + A4*R5;
  const double T4 = A2*R0 + A4*R1 + A5*R2;
  const double T5 = A2*R3 + A4*R4 + A5*R5;
  return Sym{R0*T0 + R1*T2 + R2*T4, R3*T0 + R4*T2 + R5*T4, R6*T0 + R7*T2 + R8*T4,
             R3*T1 + R4*T3 + R5*T5, R6*T1 + R7*T3 + R8*T5,
             R6*(A0*R6 + A1*R7 + A2*R8) + R7*(A1*R6 + A3*R7 + A4*R8) + R8*(A2*R6 + A4*R7 + A5*R8)};
}
// max(double, SymTensor) and min(double, SymTensor)
// (src/Geometry/GeomSymmetricTensorInline_default.hh:2286-2345): the
// eigenvalues limited, the tensor rebuilt from its eigenvectors, unless no
// eigenvalue crosses the bound.
inline Sym symMax(double maxValue, const Sym& t) {
  const Eig3 e = symEigenVectors(t);
  if (minElement(e.values) > maxValue) return t;
  const Sym d{std::max(maxValue, e.values.x), 0.0, 0.0, std::max(maxValue, e.values.y), 0.0,
              std::max(maxValue, e.values.z)};
  return rotationalTransform(d, e.vectors);
}
inline Sym symMin(double minValue, const Sym& t) {
  const Eig3 e = symEigenVectors(t);
  if (maxElement(e.values) < minValue) return t;
  const Sym d{std::min(minValue, e.values.x), 0.0, 0.0, std::min(minValue, e.values.y), 0.0,
              std::min(minValue, e.values.z)};
  return rotationalTransform(d, e.vectors);
}
inline T9 tzero() { return T9{0, 0, 0, 0, 0, 0, 0, 0, 0}; }
inline T9 dyad(const V3& a, const V3& b) {
  return T9{a.x*b.x, a.x*b.y, a.x*b.z,
            a.y*b.x, a.y*b.y, a.y*b.z,
            a.z*b.x, a.z*b.y, a.z*b.z};
}
inline T9 tmul(const T9& t, double s) {
  return T9{t.xx*s, t.xy*s, t.xz*s, t.yx*s, t.yy*s, t.yz*s, t.zx*s, t.zy*s, t.zz*s};
}
inline T9 tneg(const T9& t) { return T9{-t.xx, -t.xy, -t.xz, -t.yx, -t.yy, -t.yz, -t.zx, -t.zy, -t.zz}; }
inline void taddto(T9& a, const T9& b) {
  a.xx += b.xx; a.xy += b.xy; a.xz += b.xz; a.yx += b.yx; a.yy += b.yy; a.yz += b.yz;
  a.zx += b.zx; a.zy += b.zy; a.zz += b.zz;
}
inline void tsubfrom(T9& a, const T9& b) {
  a.xx -= b.xx; a.xy -= b.xy; a.xz -= b.xz; a.yx -= b.yx; a.yy -= b.yy; a.yz -= b.yz;
  a.zx -= b.zx; a.zy -= b.zy; a.zz -= b.zz;
}
// Tensor/double and Tensor/=double multiply by the reciprocal.
inline T9 tdiv(const T9& t, double s) { const double inv = 1.0/s; return tmul(t, inv); }
inline double tdet(const T9& t) {
  return (t.xx*t.yy*t.zz + t.xy*t.yz*t.zx + t.xz*t.yx*t.zy -
          t.xx*t.yz*t.zy - t.xy*t.yx*t.zz - t.xz*t.yy*t.zx);
}
inline T9 tinverse(const T9& t) {
  const T9 c{t.yy*t.zz - t.yz*t.zy, t.xz*t.zy - t.xy*t.zz, t.xy*t.yz - t.xz*t.yy,
             t.yz*t.zx - t.yx*t.zz, t.xx*t.zz - t.xz*t.zx, t.xz*t.yx - t.xx*t.yz,
             t.yx*t.zy - t.yy*t.zx, t.xy*t.zx - t.xx*t.zy, t.xx*t.yy - t.xy*t.yx};
  return tdiv(c, tdet(t));
}
inline T9 tdot(const T9& a, const T9& b) {
  return T9{a.xx*b.xx + a.xy*b.yx + a.xz*b.zx,
            a.xx*b.xy + a.xy*b.yy + a.xz*b.zy,
            a.xx*b.xz + a.xy*b.yz + a.xz*b.zz,
            a.yx*b.xx + a.yy*b.yx + a.yz*b.zx,
            a.yx*b.xy + a.yy*b.yy + a.yz*b.zy,
            a.yx*b.xz + a.yy*b.yz + a.yz*b.zz,
            a.zx*b.xx + a.zy*b.yx + a.zz*b.zx,
            a.zx*b.xy + a.zy*b.yy + a.zz*b.zy,
            a.zx*b.xz + a.zy*b.yz + a.zz*b.zz};
}
inline V3 tvdot(const T9& t, const V3& r) {
  return V3{t.xx*r.x + t.xy*r.y + t.xz*r.z,
            t.yx*r.x + t.yy*r.y + t.yz*r.z,
            t.zx*r.x + t.zy*r.y + t.zz*r.z};
}
inline double ttrace(const T9& t) { return t.xx + t.yy + t.zz; }
// double * Tensor::one
inline T9 tdiag(double s) { return T9{1.0*s, 0.0*s, 0.0*s, 0.0*s, 1.0*s, 0.0*s, 0.0*s, 0.0*s, 1.0*s}; }

struct Plane {
  V3 point, normal;
  Plane() : point{0, 0, 0}, normal{1, 0, 0} {}
  Plane(const V3& p, const V3& n) : point(p), normal(unitVector(n)) {}
  double signedDistance(const V3& r) const { return dot(normal, vsub(r, point)); }
  double minimumDistance(const V3& r) const { return std::abs(dot(normal, vsub(r, point))); }
  V3 closestPointOnPlane(const V3& p) const { return vadd(p, vmul(normal, dot(vsub(point, p), normal))); }
  // GeomPlane::compare: -1 if the point is above the plane, 1 below, 0 on.
  int compare(const V3& r) const {
    const double thpt = dot(normal, vsub(r, point));
    return fuzzyEqual(thpt, 0.0) ? 0 : (thpt > 0.0 ? -1 : 1);
  }
};

// src/Boundary/mapPositionThroughPlanes.hh:13-22
inline V3 mapPositionThroughPlanes(const V3& position, const Plane& enterPlane, const Plane& exitPlane) {
  const V3 p0 = exitPlane.closestPointOnPlane(position);
  const double s = enterPlane.signedDistance(position);
  return vsub(p0, vmul(exitPlane.normal, s));
}

}  // namespace orc

#endif
