// Dim<3> FP64 geometry, plane mapping and TableKernel lookups for the device.
//
// Every expression keeps the reference's operand order so that, compiled
// with -fmad=false (no FMA contraction), each per-pair quantity is
// bit-identical to the x86-64 FP64 reference:
//   GeomVector<3>          src/Geometry/GeomVectorInline_default.hh:395-575,795-975
//   GeomSymmetricTensor<3> src/Geometry/GeomSymmetricTensorInline_default.hh:895-955,1546-1661,2083-2109
//   GeomTensor<3>          src/Geometry/GeomTensorInline_default.hh:931-937,1817-1895,1918-1958
//   GeomPlane / mapPositionThroughPlanes
//                          src/Geometry/GeomPlane.cc:218-259, src/Boundary/mapPositionThroughPlanes.hh:13-22
//   TableKernel lookups    src/Kernel/TableKernelInline.hh:11-78,262-294
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define SPH_HD __host__ __device__ __forceinline__

namespace sphgpu {

struct V3 {
  double x, y, z;
};
struct Sym {
  double xx, xy, xz, yy, yz, zz;
};
struct T9 {
  double xx, xy, xz, yx, yy, yz, zx, zy, zz;
};

SPH_HD double sgn(double x) { return x < 0.0 ? -1.0 : 1.0; }
SPH_HD double dmin(double a, double b) { return b < a ? b : a; }   // std::min semantics
SPH_HD double dmax(double a, double b) { return a < b ? b : a; }   // std::max semantics
SPH_HD double dabs(double a) { return a < 0.0 ? -a : (a == 0.0 ? 0.0 : a); }
SPH_HD bool fuzzyEqual(double lhs, double rhs, double fuzz = 1.0e-15) {
  const double d = lhs - rhs;
  return dabs(d)/dmax(1.0, dabs(lhs) + dabs(rhs)) < fuzz;
}
SPH_HD double safeInv(double x, double fuzz = 1.0e-30) { return x/(x*x + fuzz); }
SPH_HD double safeInvVar(double x, double fuzz = 1.0e-30) { return sgn(x)/dmax(fuzz, dabs(x)); }

SPH_HD V3 vadd(const V3& a, const V3& b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
SPH_HD V3 vsub(const V3& a, const V3& b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
SPH_HD V3 vmul(const V3& a, double s) { return V3{a.x*s, a.y*s, a.z*s}; }
SPH_HD V3 vdiv(const V3& a, double s) { const double inv = 1.0/s; return V3{a.x*inv, a.y*inv, a.z*inv}; }
SPH_HD double dot(const V3& a, const V3& b) { return a.x*b.x + a.y*b.y + a.z*b.z; }
SPH_HD double mag2(const V3& a) { return a.x*a.x + a.y*a.y + a.z*a.z; }
SPH_HD double mag(const V3& a) { return sqrt(a.x*a.x + a.y*a.y + a.z*a.z); }
SPH_HD V3 unitVector(const V3& a) {
  const double m = mag(a);
  return m > 1.0e-50 ? vdiv(a, m) : V3{1.0, 0.0, 0.0};
}
SPH_HD double vmaxAbs(const V3& a) { return dmax(dabs(a.x), dmax(dabs(a.y), dabs(a.z))); }
SPH_HD double vmin(const V3& a) { return dmin(a.x, dmin(a.y, a.z)); }
SPH_HD double vmax(const V3& a) { return dmax(a.x, dmax(a.y, a.z)); }

SPH_HD V3 sdot(const Sym& s, const V3& r) {
  return V3{s.xx*r.x + s.xy*r.y + s.xz*r.z,
            s.xy*r.x + s.yy*r.y + s.yz*r.z,
            s.xz*r.x + s.yz*r.y + s.zz*r.z};
}
SPH_HD double sdet(const Sym& s) {
  return (s.xx*s.yy*s.zz +
          s.xy*s.yz*s.xz +
          s.xz*s.xy*s.yz -
          s.xx*s.yz*s.yz -
          s.xy*s.xy*s.zz -
          s.xz*s.yy*s.xz);
}
SPH_HD Sym smul(const Sym& s, double v) { return Sym{s.xx*v, s.xy*v, s.xz*v, s.yy*v, s.yz*v, s.zz*v}; }
SPH_HD Sym sdiv(const Sym& s, double v) { const double inv = 1.0/v; return smul(s, inv); }
SPH_HD Sym sadd(const Sym& a, const Sym& b) {
  return Sym{a.xx + b.xx, a.xy + b.xy, a.xz + b.xz, a.yy + b.yy, a.yz + b.yz, a.zz + b.zz};
}
SPH_HD Sym sneg(const Sym& a) { return Sym{-a.xx, -a.xy, -a.xz, -a.yy, -a.yz, -a.zz}; }
SPH_HD Sym selfdyad(const V3& a) {
  return Sym{a.x*a.x, a.x*a.y, a.x*a.z, a.y*a.y, a.y*a.z, a.z*a.z};
}
// H = h I exactly: then H.dot(r) = r*h bit for bit (the off-diagonal
// products are exact zeros).
SPH_HD bool isoSym(const Sym& s) {
  return s.xy == 0.0 && s.xz == 0.0 && s.yz == 0.0 && s.xx == s.yy && s.xx == s.zz;
}
// GeomSymmetricTensor<3>::Inverse (cofactors over the determinant).
SPH_HD Sym sinverse(const Sym& s) {
  const Sym c{s.yy*s.zz - s.yz*s.yz,
              s.yz*s.xz - s.xy*s.zz,
              s.xy*s.yz - s.yy*s.xz,
              s.xx*s.zz - s.xz*s.xz,
              s.xy*s.xz - s.xx*s.yz,
              s.xx*s.yy - s.xy*s.xy};
  return sdiv(c, sdet(s));
}
SPH_HD double smaxAbs(const Sym& s) {
  return dmax(dabs(s.xx), dmax(dabs(s.xy), dmax(dabs(s.xz), dmax(dabs(s.yy), dmax(dabs(s.yz), dabs(s.zz))))));
}
// Analytic eigenvalues of a symmetric 3x3 (GeomSymmetricTensor<3>::eigenValues).
// The trigonometric calls use CUDA's libm, so results can differ from glibc by
// a few ulp for anisotropic H; for an isotropic H the result is exact.
SPH_HD V3 eigenValues(const Sym& s) {
  const double onethird = 1.0/3.0;
  const double sqrt3 = 1.7320508075688772;  // std::sqrt(3.0), correctly rounded
  const double fscale = dmax(10.0*2.220446049250313e-16, smaxAbs(s));
  const double fscalei = 1.0/fscale;
  const double a00 = s.xx*fscalei, a01 = s.xy*fscalei, a02 = s.xz*fscalei;
  const double a11 = s.yy*fscalei, a12 = s.yz*fscalei, a22 = s.zz*fscalei;
  const double c0 = a00*a11*a22 + 2.0*a01*a02*a12 - a00*a12*a12 - a11*a02*a02 - a22*a01*a01;
  const double c1 = a00*a11 - a01*a01 + a00*a22 - a02*a02 + a11*a22 - a12*a12;
  const double c2 = a00 + a11 + a22;
  const double c2Div3 = c2*onethird;
  const double aDiv3 = dmin(0.0, onethird*(c1 - c2*c2Div3));
  const double mbDiv2 = 0.5*(c0 + c2Div3*(2.0*c2Div3*c2Div3 - c1));
  const double m = sqrt(-aDiv3);
  // m == +-0 (every isotropic H): the cos/sin terms are multiplied by a zero,
  // so all three eigenvalues are fscale*c2Div3 bit for bit; skip the solve
  if (m == 0.0) {
    const double e = fscale*c2Div3;
    return V3{e, e, e};
  }
  const double q = dmin(0.0, mbDiv2*mbDiv2 + aDiv3*aDiv3*aDiv3);
  const double angle = atan2(sqrt(-q), mbDiv2)*onethird;
  const double cs = cos(angle);
  const double sn = sin(angle);
  return V3{fscale*(c2Div3 + 2.0*m*cs),
            fscale*(c2Div3 - m*(cs + sqrt3*sn)),
            fscale*(c2Div3 - m*(cs - sqrt3*sn))};
}

// GeomSymmetricTensor<3>::eigenVectors (src/Geometry/GeomSymmetricTensor_default.cc:36-95):
// the tensor scaled by its largest element, elements below 1e-20 zeroed,
// the symmetric 3x3 eigenproblem solved, eigenvalues scaled back, and every
// eigenvector column normalised.  The reference hands the solve to Eigen's
// SelfAdjointEigenSolver (not available to this build); the solve here is
// cyclic Jacobi rotations (p, q) = (0,1), (0,2), (1,2) per sweep until the
// off-diagonal mass is below 1e-32 of the diagonal, eigenvalues ascending.
// Only the eigenvalue clamp of the bounded H policies uses it.
struct Eig3 {
  V3 values;
  T9 vectors;   // column c: the eigenvector of values[c]
};
SPH_HD Eig3 symEigenVectors(const Sym& s) {
  const double fscale = dmax(10.0*2.220446049250313e-16, smaxAbs(s));
  const double fscalei = 1.0/fscale;
  double A[3][3], V[3][3];
  const double e[6] = {s.xx*fscalei, s.xy*fscalei, s.xz*fscalei, s.yy*fscalei, s.yz*fscalei, s.zz*fscalei};
  double d[6];
  for (int k = 0; k < 6; ++k) d[k] = dabs(e[k]) < 1.0e-20 ? 0.0 : e[k];
  A[0][0] = d[0]; A[0][1] = d[1]; A[0][2] = d[2];
  A[1][0] = d[1]; A[1][1] = d[3]; A[1][2] = d[4];
  A[2][0] = d[2]; A[2][1] = d[4]; A[2][2] = d[5];
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) V[i][j] = i == j ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 64; ++sweep) {
    const double off = A[0][1]*A[0][1] + A[0][2]*A[0][2] + A[1][2]*A[1][2];
    const double diag = A[0][0]*A[0][0] + A[1][1]*A[1][1] + A[2][2]*A[2][2];
    if (off <= 1e-32*diag || off == 0.0) break;
#pragma unroll
    for (int p = 0; p < 2; ++p) {
#pragma unroll
      for (int q = p + 1; q < 3; ++q) {
        if (A[p][q] == 0.0) continue;
        const double theta = (A[q][q] - A[p][p])/(2.0*A[p][q]);
        const double t = (theta >= 0.0 ? 1.0 : -1.0)/(dabs(theta) + sqrt(theta*theta + 1.0));
        const double c = 1.0/sqrt(t*t + 1.0), sn = t*c;
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
  }
  int order[3] = {0, 1, 2};
  for (int i = 0; i < 3; ++i)
    for (int j = i + 1; j < 3; ++j)
      if (A[order[j]][order[j]] < A[order[i]][order[i]]) { const int t = order[i]; order[i] = order[j]; order[j] = t; }
  double B[3][3];
  for (int c = 0; c < 3; ++c) for (int r = 0; r < 3; ++r) B[r][c] = V[r][order[c]];
  Eig3 out;
  out.values = V3{A[order[0]][order[0]]*fscale, A[order[1]][order[1]]*fscale, A[order[2]][order[2]]*fscale};
  const double x1 = 1.0/sqrt(B[0][0]*B[0][0] + B[1][0]*B[1][0] + B[2][0]*B[2][0]);
  const double x2 = 1.0/sqrt(B[0][1]*B[0][1] + B[1][1]*B[1][1] + B[2][1]*B[2][1]);
  const double x3 = 1.0/sqrt(B[0][2]*B[0][2] + B[1][2]*B[1][2] + B[2][2]*B[2][2]);
  out.vectors = T9{B[0][0]*x1, B[0][1]*x2, B[0][2]*x3,
                   B[1][0]*x1, B[1][1]*x2, B[1][2]*x3,
                   B[2][0]*x1, B[2][1]*x2, B[2][2]*x3};
  return out;
}

// GeomSymmetricTensor<3>::rotationalTransform(R): R A R^T
// (src/Geometry/GeomSymmetricTensorInline_default.hh:1981-2014).
SPH_HD Sym symRotational(const Sym& a, const T9& R) {
  const double A0 = a.xx, A1 = a.xy, A2 = a.xz, A3 = a.yy, A4 = a.yz, A5 = a.zz;
  const double R0 = R.xx, R1 = R.xy, R2 = R.xz, R3 = R.yx, R4 = R.yy, R5 = R.yz, R6 = R.zx, R7 = R.zy, R8 = R.zz;
  const double T0 = A0*R0 + A1*R1 + A2*R2;
  const double T1 = A0*R3 + A1*R4 + A2*R5;
  const double T2 = A1*R0 + A3*R1 + A4*R2;
  const double T3 = A1*R3 + A3*R4 + A4*R5;
  const double T4 = A2*R0 + A4*R1 + A5*R2;
  const double T5 = A2*R3 + A4*R4 + A5*R5;
  return Sym{R0*T0 + R1*T2 + R2*T4,
             R3*T0 + R4*T2 + R5*T4,
             R6*T0 + R7*T2 + R8*T4,
             R3*T1 + R4*T3 + R5*T5,
             R6*T1 + R7*T3 + R8*T5,
             R6*(A0*R6 + A1*R7 + A2*R8) + R7*(A1*R6 + A3*R7 + A4*R8) + R8*(A2*R6 + A4*R7 + A5*R8)};
}

// min(maxValue, max(minValue, H)) of IncrementBoundedState / ReplaceBoundedState
// for SymTensor (src/DataBase/IncrementBoundedState.cc:131-133,
// ReplaceBoundedState.cc:134-136) with the eigenvalue limiters max(double,
// SymTensor) and min(double, SymTensor)
// (src/Geometry/GeomSymmetricTensorInline_default.hh:2286-2345): a tensor whose
// eigenvalues all lie on the inner side of the bound comes back unchanged,
// otherwise it is rebuilt from its eigenvectors with the eigenvalues limited.
SPH_HD Sym boundedSym(const Sym& H, double minValue, double maxValue) {
  Sym r = H;
  {
    const Eig3 e = symEigenVectors(r);
    if (!(vmin(e.values) > minValue)) {
      const Sym d{dmax(minValue, e.values.x), 0.0, 0.0, dmax(minValue, e.values.y), 0.0, dmax(minValue, e.values.z)};
      r = symRotational(d, e.vectors);
    }
  }
  {
    const Eig3 e = symEigenVectors(r);
    if (!(vmax(e.values) < maxValue)) {
      const Sym d{dmin(maxValue, e.values.x), 0.0, 0.0, dmin(maxValue, e.values.y), 0.0, dmin(maxValue, e.values.z)};
      r = symRotational(d, e.vectors);
    }
  }
  return r;
}

SPH_HD T9 dyad(const V3& a, const V3& b) {
  return T9{a.x*b.x, a.x*b.y, a.x*b.z, a.y*b.x, a.y*b.y, a.y*b.z, a.z*b.x, a.z*b.y, a.z*b.z};
}
// Tensor.dot(Vector)
SPH_HD V3 tvdot(const T9& t, const V3& r) {
  return V3{t.xx*r.x + t.xy*r.y + t.xz*r.z,
            t.yx*r.x + t.yy*r.y + t.yz*r.z,
            t.zx*r.x + t.zy*r.y + t.zz*r.z};
}
SPH_HD T9 tmul(const T9& t, double s) {
  return T9{t.xx*s, t.xy*s, t.xz*s, t.yx*s, t.yy*s, t.yz*s, t.zx*s, t.zy*s, t.zz*s};
}
SPH_HD void taddto(T9& a, const T9& b) {
  a.xx += b.xx; a.xy += b.xy; a.xz += b.xz; a.yx += b.yx; a.yy += b.yy; a.yz += b.yz;
  a.zx += b.zx; a.zy += b.zy; a.zz += b.zz;
}
SPH_HD void tsubfrom(T9& a, const T9& b) {
  a.xx -= b.xx; a.xy -= b.xy; a.xz -= b.xz; a.yx -= b.yx; a.yy -= b.yy; a.yz -= b.yz;
  a.zx -= b.zx; a.zy -= b.zy; a.zz -= b.zz;
}
SPH_HD T9 tdiv(const T9& t, double s) { const double inv = 1.0/s; return tmul(t, inv); }
SPH_HD double tdet(const T9& t) {
  return (t.xx*t.yy*t.zz + t.xy*t.yz*t.zx + t.xz*t.yx*t.zy -
          t.xx*t.yz*t.zy - t.xy*t.yx*t.zz - t.xz*t.yy*t.zx);
}
SPH_HD T9 tinverse(const T9& t) {
  const T9 c{t.yy*t.zz - t.yz*t.zy, t.xz*t.zy - t.xy*t.zz, t.xy*t.yz - t.xz*t.yy,
             t.yz*t.zx - t.yx*t.zz, t.xx*t.zz - t.xz*t.zx, t.xz*t.yx - t.xx*t.yz,
             t.yx*t.zy - t.yy*t.zx, t.xy*t.zx - t.xx*t.zy, t.xx*t.yy - t.xy*t.yx};
  return tdiv(c, tdet(t));
}
SPH_HD T9 tdot(const T9& a, const T9& b) {
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
SPH_HD double ttrace(const T9& t) { return t.xx + t.yy + t.zz; }

// GeomPlane with a unit normal.
struct PlaneD {
  V3 point, normal;
};
SPH_HD double signedDistance(const PlaneD& p, const V3& r) { return dot(p.normal, vsub(r, p.point)); }
SPH_HD double minimumDistance(const PlaneD& p, const V3& r) { return dabs(dot(p.normal, vsub(r, p.point))); }
SPH_HD V3 closestPointOnPlane(const PlaneD& p, const V3& r) {
  return vadd(r, vmul(p.normal, dot(vsub(p.point, r), p.normal)));
}
SPH_HD V3 mapPositionThroughPlanes(const V3& position, const PlaneD& enterPlane, const PlaneD& exitPlane) {
  const V3 p0 = closestPointOnPlane(exitPlane, position);
  const double s = signedDistance(enterPlane, position);
  return vsub(p0, vmul(exitPlane.normal, s));
}
// GeomPlane::compare: -1 above the plane, 1 below, 0 on it.
SPH_HD int planeCompare(const PlaneD& p, const V3& r) {
  const double thpt = dot(p.normal, vsub(r, p.point));
  return fuzzyEqual(thpt, 0.0) ? 0 : (thpt > 0.0 ? -1 : 1);
}

// One PlanarBoundary of a PeriodicBoundary pair.
struct PlanarBC {
  PlaneD enter, exit;
};

// Up to 3 periodic axes, each with its two planar boundaries (plane1 ->
// plane2, plane2 -> plane1), in the reference's application order.
struct BoxBCs {
  PlanarBC bc[6];
  int periodic[3];
};

// Position of a ghost: the root's position mapped through one planar
// boundary per axis, axes in boundary order.  `code` holds 2 bits per axis:
// 0 = not imaged on that axis, 1/2 = imaged through planar boundary 2a / 2a+1.
SPH_HD V3 ghostPosition(const BoxBCs& B, V3 r, uint32_t code) {
  for (int a = 0; a < 3; ++a) {
    const uint32_t sel = (code >> (2*a)) & 3u;
    if (sel != 0u && B.periodic[a]) {
      const PlanarBC& bc = B.bc[2*a + (sel - 1)];
      // PlanarBoundary::updateGhostNodes -> mapPosition(pos, mExitPlane, mEnterPlane)
      r = mapPositionThroughPlanes(r, bc.exit, bc.enter);
    }
  }
  return r;
}

// TableKernel<Dim<3>> packed for the device: per table point i the six
// parabolic coefficients (aK, bK, cK, aG, bG, cG).
struct TableDev {
  const double* coef;   // 6*n
  int n;
  double stepSize, extent;
};

SPH_HD void tableKernelAndGrad(const TableDev& T, double eta, double Hdet, double& W, double& gW) {
  if (eta < T.extent) {
    const double q = eta/T.stepSize;
    int lb = int(q);
    lb = lb < T.n - 1 ? lb : T.n - 1;
    const int i0 = lb < T.n - 3 ? lb : T.n - 3;
    const int i1 = i0 + 1;
    const double x = q - i0;
    const double* c = T.coef + 6*i1;
#ifdef __CUDA_ARCH__
    const double2 c01 = __ldg(reinterpret_cast<const double2*>(c));
    const double2 c23 = __ldg(reinterpret_cast<const double2*>(c + 2));
    const double2 c45 = __ldg(reinterpret_cast<const double2*>(c + 4));
#else
    const double2 c01 = make_double2(c[0], c[1]), c23 = make_double2(c[2], c[3]), c45 = make_double2(c[4], c[5]);
#endif
    W = Hdet*(c01.x + c01.y*x + c23.x*x*x);
    gW = Hdet*(c23.y + c45.x*x + c45.y*x*x);
  } else {
    W = 0.0;
    gW = 0.0;
  }
}

SPH_HD double tableKernel(const TableDev& T, double eta, double Hdet) {
  double W, gW;
  tableKernelAndGrad(T, eta, Hdet, W, gW);
  return W;
}

}  // namespace sphgpu
