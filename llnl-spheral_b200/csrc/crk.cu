// CRKSPH hydro kernels (linear order), plain FP64 form (compiled with -fmad=false).
//
// Replaces:
//   crk_moments_corrections  computeCRKSPHMoments (src/CRKSPH/computeCRKSPHMoments.cc:40-287,
//                            NodeCoupling = 1) fused with computeLinearCRKSPHCorrections
//                            (src/CRKSPH/computeCRKSPHCorrections.cc:210-283)
//   crk_eval                 CRKSPHHydroBase::evaluateDerivatives
//                            (src/CRKSPH/CRKSPHHydroBase.cc:646-1102) with
//                            CRKSPHKernelAndGradient (src/CRKSPH/CRKSPHUtilitiesInline.hh:58-129)
//   crk_sum_volume           computeCRKSPHSumVolume (src/CRKSPH/computeCRKSPHSumVolume.cc:43-127)
//   crk_sum_density          computeCRKSPHSumMassDensity (src/CRKSPH/computeCRKSPHSumMassDensity.cc:28-139)
//
// All pair loops gather over node i's ascending CSR row.  Every CRKSPH pair
// term is even or odd under i <-> j with exact FP negation, so it is formed
// from node i's side; the only order-sensitive products (0.5*w_i*w_j) are
// taken in the reference's owner order.  Self terms enter where the
// reference adds them, so node sums see the reference's summation order.
#include "problem.cuh"

namespace sphgpu {

namespace {

__device__ __forceinline__ double ldg(const double* p) { return __ldg(p); }
__device__ __forceinline__ double& el(V3& v, int i) { return (&v.x)[i]; }
__device__ __forceinline__ double el(const V3& v, int i) { return (&v.x)[i]; }
__device__ __forceinline__ double& el(T9& t, int i, int j) { return (&t.xx)[3*i + j]; }
__device__ __forceinline__ double el(const T9& t, int i, int j) { return (&t.xx)[3*i + j]; }
__device__ __forceinline__ int symIndex(int i, int j) {
  // xx xy xz / xy yy yz / xz yz zz
  return i == 0 ? j : (i == 1 ? (j == 0 ? 1 : j + 2) : (j == 0 ? 2 : (j == 1 ? 4 : 5)));
}
__device__ __forceinline__ double sel(const Sym& s, int i, int j) { return (&s.xx)[symIndex(i, j)]; }

struct CRec {
  V3 r, v;
  double m, rho, cs, P, Hdet, vol;
  Sym H;
  double A;
  V3 B, gA;
  T9 gB;
};

__device__ __forceinline__ CRec loadCRec(const double* crec, int64_t k) {
  const double2* q = reinterpret_cast<const double2*>(crec + k*CRECW);
  double2 a[17];
#pragma unroll
  for (int t = 0; t < 17; ++t) a[t] = __ldg(q + t);
  const double* d = reinterpret_cast<const double*>(a);
  CRec R;
  R.r = V3{d[C_X], d[C_Y], d[C_Z]};
  R.v = V3{d[C_VX], d[C_VY], d[C_VZ]};
  R.m = d[C_M]; R.rho = d[C_RHO]; R.cs = d[C_CS]; R.P = d[C_P]; R.Hdet = d[C_HDET]; R.vol = d[C_VOL];
  R.H = Sym{d[C_H], d[C_H + 1], d[C_H + 2], d[C_H + 3], d[C_H + 4], d[C_H + 5]};
  R.A = d[C_A];
  R.B = V3{d[C_B], d[C_B + 1], d[C_B + 2]};
  R.gA = V3{d[C_GRADA], d[C_GRADA + 1], d[C_GRADA + 2]};
  R.gB = T9{d[C_GRADB], d[C_GRADB + 1], d[C_GRADB + 2], d[C_GRADB + 3], d[C_GRADB + 4], d[C_GRADB + 5],
            d[C_GRADB + 6], d[C_GRADB + 7], d[C_GRADB + 8]};
  return R;
}

__global__ void __launch_bounds__(256) pack_crk_records_kernel(const Member* mem, BlockMap bm) {
  const MemberBlock mb = memberBlock(bm);
  const Member& MB = mem[mb.m];
  const int64_t n = MB.n;
  const double* S = MB.S;
  const double* K = MB.K;
  const BoxBCs& bcs = MB.prm.bcs;
  const int32_t* groot = MB.groot;
  const uint32_t* gcode = MB.gcode;
  double* crec = MB.crec;
  {
    const int64_t k = mb.block*blockDim.x + threadIdx.x;
    if (k >= n + scalI(MB.scal, SC_G)) return;
    const int64_t r = k < n ? k : groot[k - n];
    V3 x{S[S_X*n + r], S[S_Y*n + r], S[S_Z*n + r]};
    if (k >= n) x = ghostPosition(bcs, x, gcode[k - n]);
    const Sym H{S[(S_H + 0)*n + r], S[(S_H + 1)*n + r], S[(S_H + 2)*n + r],
                S[(S_H + 3)*n + r], S[(S_H + 4)*n + r], S[(S_H + 5)*n + r]};
    double v[CRECW];
    v[C_X] = x.x; v[C_Y] = x.y; v[C_Z] = x.z;
    v[C_VX] = S[S_VX*n + r]; v[C_VY] = S[S_VY*n + r]; v[C_VZ] = S[S_VZ*n + r];
    v[C_M] = S[S_M*n + r]; v[C_RHO] = S[S_RHO*n + r]; v[C_CS] = S[S_CS*n + r]; v[C_P] = S[S_P*n + r];
    v[C_HDET] = sdet(H); v[C_VOL] = S[S_VOL*n + r];
    v[C_H] = H.xx; v[C_H + 1] = H.xy; v[C_H + 2] = H.xz; v[C_H + 3] = H.yy; v[C_H + 4] = H.yz; v[C_H + 5] = H.zz;
    v[C_A] = K[K_A*n + r];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      v[C_B + c] = K[(K_B + c)*n + r];
      v[C_GRADA + c] = K[(K_GRADA + c)*n + r];
    }
#pragma unroll
    for (int c = 0; c < 9; ++c) v[C_GRADB + c] = K[(K_GRADB + c)*n + r];
    double2* q = reinterpret_cast<double2*>(crec + k*CRECW);
#pragma unroll
    for (int t = 0; t < CRECW/2; ++t) q[t] = make_double2(v[2*t], v[2*t + 1]);
  }
}

// Record fields shared with the SPH record (positions, H, Hdet).
__device__ __forceinline__ V3 recPos(const double* rec, int64_t j) {
  return V3{ldg(rec + j*RECW + R_X), ldg(rec + j*RECW + R_Y), ldg(rec + j*RECW + R_Z)};
}
__device__ __forceinline__ Sym recH(const double* rec, int64_t j) {
  const double* h = rec + j*RECW + R_H;
  return Sym{ldg(h), ldg(h + 1), ldg(h + 2), ldg(h + 3), ldg(h + 4), ldg(h + 5)};
}

// ---------------------------------------------------------------- volumes
__global__ void __launch_bounds__(128) crk_sum_volume_kernel(const Member* mem, BlockMap bm) {
  const MemberBlock mb = memberBlock(bm);
  const Member& MB = mem[mb.m];
  const int64_t n = MB.n;
  const int64_t i = mb.block*blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Params& P = MB.prm;
  const double* rec = MB.rec;
  const int64_t* offsets = MB.offsets;
  const int32_t* nbr = MB.nbr;
  double* S = MB.S;
  const V3 ri = recPos(rec, i);
  const Sym Hi = recH(rec, i);
  const double Hdeti = ldg(rec + i*RECW + R_HDET);
  const double half = 0.5*P.W.extent;
  const double etaVolMax = half*half*half*(4.0/3.0*3.14159265358979323846);
  double vol = 0.0;
  for (int64_t k = offsets[i]; k < offsets[i + 1]; ++k) {
    const int32_t j = __ldg(nbr + k);
    const V3 rij = vsub(ri, recPos(rec, j));
    vol += tableKernel(P.W, mag(sdot(Hi, rij)), Hdeti);
  }
  vol += tableKernel(P.W, 0.0, Hdeti);
  S[S_VOL*n + i] = dmin(etaVolMax/Hdeti, 1.0/vol);
}

__global__ void __launch_bounds__(256) crk_volume_from_density_kernel(const Member* mem, BlockMap bm) {
  const MemberBlock mb = memberBlock(bm);
  const Member& MB = mem[mb.m];
  const int64_t n = MB.n;
  const int64_t i = mb.block*blockDim.x + threadIdx.x;
  if (i >= n) return;
  double* S = MB.S;
  // mass/massDensity as the reference's FieldList quotient forms it: times
  // safeInvVar(rho, 1e-60) (src/Field/FieldInline.hh:614-623,
  // src/Utilities/safeInv.hh:24-27), not a division.
  const double rho = S[S_RHO*n + i];
  const double s = rho > 0.0 ? 1.0 : (rho < 0.0 ? -1.0 : 0.0);
  S[S_VOL*n + i] = S[S_M*n + i]*(s/fmax(1.0e-60, fabs(rho)));
}

__global__ void __launch_bounds__(128) crk_sum_density_kernel(const Member* mem, BlockMap bm) {
  const MemberBlock mb = memberBlock(bm);
  const Member& MB = mem[mb.m];
  const int64_t n = MB.n;
  const int64_t i = mb.block*blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Params& P = MB.prm;
  const double* rec = MB.rec;
  const int64_t* offsets = MB.offsets;
  const int32_t* nbr = MB.nbr;
  const int32_t* groot = MB.groot;
  double* S = MB.S;
  const double mi = S[S_M*n + i], Vi = S[S_VOL*n + i];
  const double Hdeti = ldg(rec + i*RECW + R_HDET);
  const V3 ri = recPos(rec, i);
  double wsum = 0.0, rho = 0.0, vol1 = 0.0;
  for (int64_t k = offsets[i]; k < offsets[i + 1]; ++k) {
    const int32_t j = __ldg(nbr + k);
    const int64_t r = j < n ? (int64_t)j : (int64_t)__ldg(groot + (j - n));
    const double mj = ldg(S + S_M*n + r), Vj = ldg(S + S_VOL*n + r);
    const V3 rij = vsub(ri, recPos(rec, j));
    const double Wj = tableKernel(P.W, mag(sdot(recH(rec, j), rij)), ldg(rec + (int64_t)j*RECW + R_HDET));
    wsum += Vj*Wj;
    rho += mj*Vj*Wj;
    vol1 += Vj*Vj*Wj;
  }
  const double W0 = tableKernel(P.W, 0.0, Hdeti);
  wsum += Vi*W0;
  vol1 = (vol1 + Vi*Vi*W0)/wsum;
  S[S_RHO*n + i] = dmax(dmax(P.rhoMin, 0.1*mi*Hdeti), dmin(P.rhoMax, (rho + mi*Vi*W0)/(wsum*vol1)));
}

// ---------------------------------------------------------------- moments + corrections
__global__ void __launch_bounds__(128) crk_moments_corrections_kernel(const Member* mem, BlockMap bm) {
  const MemberBlock mb = memberBlock(bm);
  const Member& MB = mem[mb.m];
  const int64_t n = MB.n;
  const int64_t i = mb.block*blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Params& P = MB.prm;
  const double* rec = MB.rec;
  const int64_t* offsets = MB.offsets;
  const int32_t* nbr = MB.nbr;
  const int32_t* groot = MB.groot;
  const double* S = MB.S;
  double* K = MB.K;
  const V3 ri = recPos(rec, i);
  const Sym Hi = recH(rec, i);
  const double Hdeti = ldg(rec + i*RECW + R_HDET);
  const double wi = S[S_VOL*n + i];
  double m0 = 0.0;
  V3 m1{0, 0, 0}, gm0{0, 0, 0};
  double m2[6] = {0, 0, 0, 0, 0, 0};
  T9 gm1{0, 0, 0, 0, 0, 0, 0, 0, 0};
  double gm2[27];
#pragma unroll
  for (int c = 0; c < 27; ++c) gm2[c] = 0.0;
  const double wwself = wi*tableKernel(P.W, 0.0, Hdeti);
  bool selfDone = false;
  const int64_t k0 = offsets[i], k1 = offsets[i + 1];
  for (int64_t k = k0; k <= k1; ++k) {
    const int32_t j = k < k1 ? __ldg(nbr + k) : INT32_MAX;
    if (!selfDone && j > (int32_t)i) {
      m0 += wwself;
      gm1.xx += 1.0*wwself; gm1.xy += 0.0*wwself; gm1.xz += 0.0*wwself;
      gm1.yx += 0.0*wwself; gm1.yy += 1.0*wwself; gm1.yz += 0.0*wwself;
      gm1.zx += 0.0*wwself; gm1.zy += 0.0*wwself; gm1.zz += 1.0*wwself;
      selfDone = true;
    }
    if (k == k1) break;
    const int64_t r = j < n ? (int64_t)j : (int64_t)__ldg(groot + (j - n));
    const double wj = ldg(S + S_VOL*n + r);
    const V3 rij = vsub(ri, recPos(rec, j));
    const Sym Hj = recH(rec, j);
    const double Hdetj = ldg(rec + (int64_t)j*RECW + R_HDET);
    const V3 etai = sdot(Hi, rij);
    const V3 etaj = sdot(Hj, rij);
    double Wa, gWa, Wb, gWb;
    tableKernelAndGrad(P.W, mag(etai), Hdeti, Wa, gWa);
    tableKernelAndGrad(P.W, mag(etaj), Hdetj, Wb, gWb);
    const double Wij = 0.5*(Wa + Wb);
    const V3 gradWj = vmul(vadd(vmul(sdot(Hj, unitVector(etaj)), gWb), vmul(sdot(Hi, unitVector(etai)), gWa)), 0.5);
    const double wwj = wj*Wij;
    m0 += wwj;
#pragma unroll
    for (int ii = 0; ii < 3; ++ii) el(gm0, ii) += wj*el(gradWj, ii);
#pragma unroll
    for (int ii = 0; ii < 3; ++ii) {
      el(m1, ii) += wwj*el(rij, ii);
#pragma unroll
      for (int jj = 0; jj < 3; ++jj) el(gm1, ii, jj) += wj*el(rij, ii)*el(gradWj, jj);
      el(gm1, ii, ii) += wj*Wij;
    }
#pragma unroll
    for (int ii = 0; ii < 3; ++ii) {
#pragma unroll
      for (int jj = ii; jj < 3; ++jj) m2[symIndex(ii, jj)] += wwj*(el(rij, ii)*el(rij, jj));
#pragma unroll
      for (int jj = 0; jj < 3; ++jj) {
        const double thpt = el(rij, ii)*el(rij, jj);
#pragma unroll
        for (int kk = 0; kk < 3; ++kk) gm2[9*ii + 3*jj + kk] += wj*thpt*el(gradWj, kk);
        gm2[9*ii + 3*jj + jj] += wwj*el(rij, ii);
        gm2[9*jj + 3*ii + jj] += wwj*el(rij, ii);
      }
    }
  }
  // computeLinearCRKSPHCorrections
  const Sym m2s{m2[0], m2[1], m2[2], m2[3], m2[4], m2[5]};
  const double hdet2 = 1.0/(Hdeti*Hdeti);
  const double m2det = sdet(m2s);
  Sym m2inv{0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  if (fabs(m2det) > 1.0e-5*hdet2) {
    const Sym c{m2s.yy*m2s.zz - m2s.yz*m2s.yz, m2s.yz*m2s.xz - m2s.xy*m2s.zz, m2s.xy*m2s.yz - m2s.yy*m2s.xz,
                m2s.xx*m2s.zz - m2s.xz*m2s.xz, m2s.xy*m2s.xz - m2s.xx*m2s.yz, m2s.xx*m2s.yy - m2s.xy*m2s.xy};
    m2inv = sdiv(c, m2det);
  }
  const V3 m2invm1 = sdot(m2inv, m1);
  const double Ainv = m0 - dot(m2invm1, m1);
  const double A = 1.0/Ainv;
  const V3 B{-m2invm1.x, -m2invm1.y, -m2invm1.z};
  V3 gA = vmul(gm0, -A*A);
  T9 gB{0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int ii = 0; ii < 3; ++ii) {
    for (int jj = 0; jj < 3; ++jj) {
      for (int kk = 0; kk < 3; ++kk) {
        el(gA, ii) += A*A*sel(m2inv, jj, kk)*el(m1, kk)*el(gm1, jj, ii);
        el(gA, ii) += A*A*sel(m2inv, jj, kk)*el(gm1, kk, ii)*el(m1, jj);
        el(gB, ii, jj) -= sel(m2inv, ii, kk)*el(gm1, kk, jj);
        for (int ll = 0; ll < 3; ++ll) {
          for (int mm = 0; mm < 3; ++mm) {
            el(gA, ii) -= A*A*sel(m2inv, jj, kk)*gm2[9*kk + 3*ll + ii]*sel(m2inv, ll, mm)*el(m1, mm)*el(m1, jj);
            el(gB, ii, jj) += sel(m2inv, ii, kk)*gm2[9*kk + 3*ll + jj]*sel(m2inv, ll, mm)*el(m1, mm);
          }
        }
      }
    }
  }
  double* o = K + i;
  o[K_A*n] = A;
  for (int c = 0; c < 3; ++c) {
    o[(K_B + c)*n] = el(B, c);
    o[(K_GRADA + c)*n] = el(gA, c);
    o[(K_M1 + c)*n] = el(m1, c);
    o[(K_GRADM0 + c)*n] = el(gm0, c);
  }
  for (int c = 0; c < 9; ++c) {
    o[(K_GRADB + c)*n] = (&gB.xx)[c];
    o[(K_GRADM1 + c)*n] = (&gm1.xx)[c];
  }
  o[K_M0*n] = m0;
  for (int c = 0; c < 6; ++c) o[(K_M2 + c)*n] = m2[c];
  for (int c = 0; c < 27; ++c) o[(K_GRADM2 + c)*n] = gm2[c];
}

// CRKSPHKernelAndGradient, LinearOrder (correction limits at +-max never bind).
__device__ __forceinline__ void crkKernel(const TableDev& T, const V3& rij, const V3& etai, const Sym& Hi,
                                          double Hdeti, const V3& etaj, const Sym& Hj, double Hdetj, double Ai,
                                          const V3& Bi, const V3& gradAi, const T9& gradBi, double& WCRK,
                                          double& gradWSPH, V3& gradWCRK) {
  double Wa, gWa, Wb, gWb;
  tableKernelAndGrad(T, mag(etai), Hdeti, Wa, gWa);
  tableKernelAndGrad(T, mag(etaj), Hdetj, Wb, gWb);
  const double Wij = 0.5*(Wa + Wb);
  const V3 gradWij = vmul(vadd(vmul(sdot(Hi, unitVector(etai)), gWa), vmul(sdot(Hj, unitVector(etaj)), gWb)), 0.5);
  gradWSPH = 0.5*(gWa + gWb);
  const double correction0 = Ai*(1.0 + dot(Bi, rij));
  const double correction = dmax(-1.7976931348623157e308, dmin(1.7976931348623157e308, correction0));
  WCRK = correction*Wij;
  gradWCRK = vmul(gradWij, correction);
  if (correction0 > -1.7976931348623157e308 && correction0 < 1.7976931348623157e308) {
    gradWCRK = vadd(gradWCRK, vadd(vmul(vmul(Bi, Ai), Wij), vmul(vmul(gradAi, 1.0 + dot(Bi, rij)), Wij)));
#pragma unroll
    for (int ii = 0; ii < 3; ++ii)
#pragma unroll
      for (int jj = 0; jj < 3; ++jj) el(gradWCRK, ii) += Ai*Wij*el(gradBi, jj, ii)*el(rij, jj);
  }
}

// CRKSPHMonaghanGingoldViscosity::Piij
// (src/ArtificialViscosity/CRKSPHMonaghanGingoldViscosity.cc:188-262): the
// velocity difference the Q sees.  The cached velocity gradients of both
// nodes are projected onto half the separation; their ratio feeds the van
// Leer limiter, which is released toward the full Q for pairs closer than
// etaCrit.  The velocities are then reconstructed to the midpoint.  Every
// term is even under i <-> j or flips sign exactly with it, so forming it
// from node i's side gives the owner-oriented value of the reference, up to
// the sign that the orientation-invariant mu absorbs.
__device__ __forceinline__ double limiterVL(double x) {
  return x > 0.0 ? 2.0/(1.0 + x)*2.0*x/(1.0 + x) : 0.0;                   // van Leer
}

__device__ __forceinline__ T9 loadQGrad(const double* qgrad, int64_t r) {
  const double2* q = reinterpret_cast<const double2*>(qgrad + r*QGRADW);
  const double2 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2), d = __ldg(q + 3), e = __ldg(q + 4);
  return T9{a.x, a.y, b.x, b.y, c.x, c.y, d.x, d.y, e.x};
}

__device__ __forceinline__ V3 crkQVelocityDifference(const Params& P, const T9& Gi, const T9& Gj, const V3& ri,
                                                     const V3& rj, const V3& vi, const V3& vj, const V3& etai,
                                                     const V3& etaj) {
  const V3 xij = vmul(vsub(ri, rj), 0.5);
  const double gradi = dot(tvdot(Gi, xij), xij);
  const double gradj = dot(tvdot(Gj, xij), xij);
  const double rI = gradi/(sgn(gradj)*dmax(1.0e-30, dabs(gradj)));
  const double rJ = gradj/(sgn(gradi)*dmax(1.0e-30, dabs(gradi)));
  double phi = limiterVL(dmin(rI, rJ));
  const double etaij = dmin(mag(etai), mag(etaj));
  if (etaij < P.etaCrit) {
    const double y = (etaij - P.etaCrit)/P.etaFold;
    phi *= exp(-(y*y));
  }
  const V3 vi1 = vsub(vi, tvdot(tmul(Gi, phi), xij));
  const V3 vj1 = vadd(vj, tvdot(tmul(Gj, phi), xij));
  return vsub(vi1, vj1);
}

// The velocity gradient the CRKSPH Q caches at initialize (the previous
// evaluation's), as [n][QGRADW] records.
__global__ void __launch_bounds__(256) crk_qgrad_kernel(const Member* mem, BlockMap bm) {
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const int64_t i = mb.block*blockDim.x + threadIdx.x;
  if (i >= M.n) return;
  double* q = M.qgrad + i*QGRADW;
#pragma unroll
  for (int c = 0; c < 9; ++c) q[c] = M.D[(D_DVDX + c)*M.n + i];
  q[9] = 0.0;
}

template<bool XSPH, bool COMPAT, bool SOLO, bool QCRK>
__global__ void __launch_bounds__(128) crk_eval_kernel(const Member* mem, BlockMap bm, const Member single) {
  const MemberBlock mb = memberBlock(bm);
  const Member& MB = SOLO ? single : mem[mb.m];   // one member: read from the kernel parameters
  const int64_t n = MB.n;
  const int64_t i = mb.block*blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Params& P = MB.prm;
  const double* crec = MB.crec;
  const int64_t* offsets = MB.offsets;
  const int32_t* nbr = MB.nbr;
  double* D = MB.D;
  double* K = MB.K;
  double* pacc = MB.pacc;
  const int64_t ecap = MB.ecap;
  const CRec I = loadCRec(crec, i);
  const double Cl = P.Cl*(0.5*(1.0 + 1.0)*1.0);
  const double Cq = P.Cq*(0.5*(1.0 + 1.0)*1.0);
  double wns = 0.0, maxvp = 0.0, effvp = 0.0, viscW = 0.0, DepsDt = 0.0;
  V3 DvDt{0, 0, 0}, gradRho{0, 0, 0}, XSPHdv{0, 0, 0};
  Sym m2{0, 0, 0, 0, 0, 0};
  T9 DvDx{0, 0, 0, 0, 0, 0, 0, 0, 0};
  const int64_t k0 = offsets[i], k1 = offsets[i + 1];
  for (int64_t k = k0; k < k1; ++k) {
    const int32_t j = __ldg(nbr + k);
    const CRec J = loadCRec(crec, j);
    const bool own = j > (int32_t)i;
    const V3 rij = vsub(I.r, J.r);
    const V3 etai = sdot(I.H, rij);
    const V3 etaj = sdot(J.H, rij);
    const V3 vij = vsub(I.v, J.v);
    V3 vQ = vij;
    if (QCRK) {
      const int64_t rootj = j < n ? (int64_t)j : (int64_t)__ldg(MB.groot + (j - n));
      vQ = crkQVelocityDifference(P, loadQGrad(MB.qgrad, i), loadQGrad(MB.qgrad, rootj), I.r, J.r, I.v, J.v,
                                  etai, etaj);
    }
    double Wj, gWj, Wi, gWi;
    V3 gradWj, gradWi;
    crkKernel(P.W, rij, etai, I.H, I.Hdet, etaj, J.H, J.Hdet, I.A, I.B, I.gA, I.gB, Wj, gWj, gradWj);
    crkKernel(P.W, V3{-rij.x, -rij.y, -rij.z}, V3{-etaj.x, -etaj.y, -etaj.z}, J.H, J.Hdet,
              V3{-etai.x, -etai.y, -etai.z}, I.H, I.Hdet, J.A, J.B, J.gA, J.gB, Wi, gWi, gradWi);
    const V3 deltagrad = vsub(gradWj, gradWi);
    // SPH moments for the ideal H
    {
      double W0a, gW0a;
      tableKernelAndGrad(P.W, mag(etai), I.Hdet, W0a, gW0a);
      const V3 gradWSPHi = vmul(sdot(I.H, unitVector(etai)), gW0a);
      const double rij2 = mag2(rij);
      const Sym thpt = smul(selfdyad(rij), safeInvVar(rij2*rij2*rij2));
      wns += 1.0*fabs(gWi);
      m2 = sadd(m2, smul(thpt, 1.0*mag2(gradWSPHi)));
    }
    // Monaghan-Gingold Pi (orientation-invariant mu)
    const double mui = dot(vQ, etai)/(mag2(etai) + P.eps2);
    const double muj = dot(vQ, etaj)/(mag2(etaj) + P.eps2);
    const double mi0 = dmin(0.0, mui), mj0 = dmin(0.0, muj);
    const double ei = -Cl*I.cs*(P.linearInExp ? mui : mi0) + Cq*(P.quadInExp ? -sgn(mui)*mui*mui : mi0*mi0);
    const double ej = -Cl*J.cs*(P.linearInExp ? muj : mj0) + Cq*(P.quadInExp ? -sgn(muj)*muj*muj : mj0*mj0);
    const double qi = ei/I.rho, qj = ej/J.rho;
    // (rho_i^2 Pi_i + rho_j^2 Pi_j).dot(deltagrad): owner term first
    const double qsi = qi*(I.rho*I.rho), qsj = qj*(J.rho*J.rho);
    const double qsum = own ? qsi + qsj : qsj + qsi;
    const V3 Qacc = vmul(deltagrad, qsum);
    const double workQi = J.rho*J.rho*dot(vmul(vij, qj), deltagrad);
    const double Qi = I.rho*I.rho*fabs(qi);
    maxvp = dmax(maxvp, 4.0*Qi);
    effvp += J.vol*Qi*Wj;
    const double f = own ? 0.5*I.vol*J.vol : 0.5*J.vol*I.vol;    // 0.5*weight_owner*weight_other
    viscW += f/I.m*workQi;
    tsubfrom(DvDx, tmul(dyad(vij, gradWj), J.vol));
    gradRho = vadd(gradRho, vmul(gradWj, J.vol*(J.rho - I.rho)));
    const double Psum = own ? I.P + J.P : J.P + I.P;
    const V3 force = vmul(vadd(vmul(deltagrad, Psum), Qacc), f);
    DvDt = vsub(DvDt, vdiv(force, I.m));
    if (COMPAT) {
      // owner's pair acceleration (-force_owner/m_owner)
      const V3 pa = own ? vdiv(V3{-force.x, -force.y, -force.z}, I.m) : vdiv(force, J.m);
      pacc[k] = pa.x;
      pacc[ecap + k] = pa.y;
      pacc[2*ecap + k] = pa.z;
    }
    DepsDt += f*(J.P*dot(vij, deltagrad) + workQi)/I.m;
    if (XSPH) XSPHdv = vsub(XSPHdv, vmul(vij, J.vol*Wj));
  }
  // ---- per-node finish (src/CRKSPH/CRKSPHHydroBase.cc:1036-1081)
  const double DrhoDt = -I.rho*ttrace(DvDx);
  wns = dmax(0.0, wns/I.Hdet);
  wns = sgn(wns)*pow(fabs(wns), 0.3333333333333333);
  m2 = sdiv(m2, I.Hdet*I.Hdet);
  const V3 DxDt = XSPH ? vadd(I.v, XSPHdv) : I.v;
  const Sym DHDt = smul(sdiv(sneg(I.H), 3.0), ttrace(DvDx));
  double nPerhCur;
  if (fuzzyEqual(wns, 0.0)) {
    nPerhCur = 0.5*P.nPerh;
  } else {
    nPerhCur = equivalentNodesPerSmoothingScale(P, wns);
  }
  const double s = dmin(4.0, dmax(0.25, P.nPerh/(nPerhCur + 1.0e-30)));
  const double a = s < 1.0 ? 0.4*(1.0 + s*s) : 0.4*(1.0 + 1.0/(s*s*s));
  const double hi1 = dmin(P.hmax, dmax(P.hmin, (1.0/I.H.xx)*(1.0 - a + a*s)));
  const double hinv = 1.0/hi1;

  double* d = D + i;
  d[(D_DXDT + 0)*n] = DxDt.x; d[(D_DXDT + 1)*n] = DxDt.y; d[(D_DXDT + 2)*n] = DxDt.z;
  d[(D_DVDT + 0)*n] = DvDt.x; d[(D_DVDT + 1)*n] = DvDt.y; d[(D_DVDT + 2)*n] = DvDt.z;
  d[D_DRHODT*n] = DrhoDt;
  d[D_DEPSDT*n] = DepsDt;
  d[(D_DHDT + 0)*n] = DHDt.xx; d[(D_DHDT + 1)*n] = DHDt.xy; d[(D_DHDT + 2)*n] = DHDt.xz;
  d[(D_DHDT + 3)*n] = DHDt.yy; d[(D_DHDT + 4)*n] = DHDt.yz; d[(D_DHDT + 5)*n] = DHDt.zz;
  d[(D_HIDEAL + 0)*n] = 1.0*hinv; d[(D_HIDEAL + 1)*n] = 0.0*hinv; d[(D_HIDEAL + 2)*n] = 0.0*hinv;
  d[(D_HIDEAL + 3)*n] = 1.0*hinv; d[(D_HIDEAL + 4)*n] = 0.0*hinv; d[(D_HIDEAL + 5)*n] = 1.0*hinv;
  const double* dv = &DvDx.xx;
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    d[(D_DVDX + c)*n] = dv[c];
  }
  d[D_WNS*n] = wns;
  d[(D_M2 + 0)*n] = m2.xx; d[(D_M2 + 1)*n] = m2.xy; d[(D_M2 + 2)*n] = m2.xz;
  d[(D_M2 + 3)*n] = m2.yy; d[(D_M2 + 4)*n] = m2.yz; d[(D_M2 + 5)*n] = m2.zz;
  d[(D_XSPHDV + 0)*n] = XSPHdv.x; d[(D_XSPHDV + 1)*n] = XSPHdv.y; d[(D_XSPHDV + 2)*n] = XSPHdv.z;
  d[D_MAXVP*n] = maxvp;
  d[D_EFFVP*n] = effvp;
  d[D_VISCW*n] = viscW;
  K[(K_GRADRHO + 0)*n + i] = gradRho.x;
  K[(K_GRADRHO + 1)*n + i] = gradRho.y;
  K[(K_GRADRHO + 2)*n + i] = gradRho.z;
}

}  // namespace

int crk_prepare(Batch& b) {
  for (Problem* pp : b.mem) {
    Problem& p = *pp;
    if (p.prm.hydro != SPHGPU_HYDRO_CRKSPH) continue;
    if (p.K == nullptr) {
      if (dev_alloc(reinterpret_cast<void**>(&p.K), sizeof(double)*NCRK*(size_t)p.n) != cudaSuccess) {
        set_error("CRKSPH field allocation failed");
        return SPHGPU_ERR_NOMEM;
      }
      cudaMemsetAsync(p.K, 0, sizeof(double)*NCRK*(size_t)p.n, b.stream);
      b.memDirty = true;
    }
    if (p.prm.qType == SPHGPU_Q_CRKSPH_MONAGHAN_GINGOLD && p.qgrad == nullptr) {
      if (dev_alloc(reinterpret_cast<void**>(&p.qgrad), sizeof(double)*QGRADW*(size_t)p.n) != cudaSuccess) {
        p.qgrad = nullptr;
        set_error("CRKSPH Q gradient allocation failed");
        return SPHGPU_ERR_NOMEM;
      }
      cudaMemsetAsync(p.qgrad, 0, sizeof(double)*QGRADW*(size_t)p.n, b.stream);
      b.memDirty = true;
    }
    if (p.candcap > p.creccap) {
      cudaStreamSynchronize(b.stream);
      dev_free(p.crec);
      p.crec = nullptr;
      if (dev_alloc(reinterpret_cast<void**>(&p.crec), sizeof(double)*CRECW*(size_t)p.candcap) != cudaSuccess) {
        p.creccap = 0;
        set_error("CRKSPH record allocation failed");
        return SPHGPU_ERR_NOMEM;
      }
      p.creccap = p.candcap;
      b.memDirty = true;
    }
  }
  if (b.memDirty) SPH_TRY(batch_upload(b));
  return SPHGPU_OK;
}

namespace {

bool isCrk(const Problem& p) { return p.prm.hydro == SPHGPU_HYDRO_CRKSPH; }
bool isCrkFp64(const Problem& p) { return isCrk(p) && p.cfg.precision == SPHGPU_PRECISION_FP64; }

int crk_nodes(Batch& b, int threads, BlockMap* bm, unsigned* grid, bool (*pred)(const Problem&)) {
  return batch_map_items(b, [&](const Problem& p) { return pred(p) ? p.n : (int64_t)0; }, threads, bm, grid);
}

bool crkSumVolume(const Problem& p) { return isCrk(p) && p.cfg.crkVolumeType == SPHGPU_CRK_SUMVOLUME; }
bool crkMassOverDensity(const Problem& p) { return isCrk(p) && p.cfg.crkVolumeType != SPHGPU_CRK_SUMVOLUME; }
bool crkSumDensity(const Problem& p) { return isCrk(p) && p.prm.densityUpdate == SPHGPU_DENSITY_RIGOROUS_SUM; }
bool crkQ(const Problem& p) { return isCrk(p) && p.prm.qType == SPHGPU_Q_CRKSPH_MONAGHAN_GINGOLD; }

}  // namespace

int launch_crk_sum_volume(Batch& b, bool startupOnly) {
  BlockMap bm;
  unsigned grid = 0;
  SPH_TRY(batch_map_items(b, [&](const Problem& p) {
    return crkSumVolume(p) && !(startupOnly && p.crkVolumeReady) ? p.n : (int64_t)0; }, 128, &bm, &grid));
  if (grid) { crk_sum_volume_kernel<<<grid, 128, 0, b.stream>>>(b.d_mem, bm); batch_count_launch(b); }
  return cuda_status(cudaGetLastError(), "CRK sum volume");
}

int launch_crk_volume_from_density(Batch& b, bool startupOnly) {
  BlockMap bm;
  unsigned grid = 0;
  SPH_TRY(batch_map_items(b, [&](const Problem& p) {
    return crkMassOverDensity(p) && !(startupOnly && p.crkVolumeReady) ? p.n : (int64_t)0; }, 256, &bm, &grid));
  if (grid) { crk_volume_from_density_kernel<<<grid, 256, 0, b.stream>>>(b.d_mem, bm); batch_count_launch(b); }
  return cuda_status(cudaGetLastError(), "CRK volume");
}

int launch_crk_sum_density(Batch& b) {
  BlockMap bm;
  unsigned grid = 0;
  SPH_TRY(crk_nodes(b, 128, &bm, &grid, crkSumDensity));
  if (grid) { crk_sum_density_kernel<<<grid, 128, 0, b.stream>>>(b.d_mem, bm); batch_count_launch(b); }
  return cuda_status(cudaGetLastError(), "CRK sum density");
}

int launch_crk_initialize(Batch& b) {
  BlockMap bm;
  unsigned grid = 0;
  SPH_TRY(crk_nodes(b, 128, &bm, &grid, isCrk));
  if (grid) { crk_moments_corrections_kernel<<<grid, 128, 0, b.stream>>>(b.d_mem, bm); batch_count_launch(b); }
  // CRKSPHMonaghanGingoldViscosity::initialize caches the last velocity gradient
  SPH_TRY(crk_nodes(b, 256, &bm, &grid, crkQ));
  if (grid) { crk_qgrad_kernel<<<grid, 256, 0, b.stream>>>(b.d_mem, bm); batch_count_launch(b); }
  return cuda_status(cudaGetLastError(), "CRK moments");
}

int launch_crk_eval(Batch& b) {
  BlockMap bm;
  unsigned grid = 0;
  SPH_TRY(batch_map_items(b, [&](const Problem& p) { return isCrkFp64(p) ? (b.capacityGrids ? p.candcap : p.n + p.G) : (int64_t)0; }, 256, &bm, &grid));
  if (grid) { pack_crk_records_kernel<<<grid, 256, 0, b.stream>>>(b.d_mem, bm); batch_count_launch(b); }
  auto key = [](const Problem& p) {
    return (crkQ(p) ? 4 : 0) | (p.prm.XSPH ? 2 : 0) | (p.prm.compatible ? 1 : 0);
  };
  const bool solo = b.mem.size() == 1;
  const Member one = solo ? describe_member(*b.mem[0]) : Member{};
  bool present[8] = {false, false, false, false, false, false, false, false};
  for (Problem* p : b.mem) if (isCrkFp64(*p)) present[key(*p)] = true;
  for (int v = 0; v < 8; ++v) {
    if (!present[v]) continue;
    SPH_TRY(batch_map_items(b, [&](const Problem& p) { return isCrkFp64(p) && key(p) == v ? p.n : (int64_t)0; }, b.evalThreads,
                            &bm, &grid));
    if (!grid) continue;
#define CRK_LAUNCH(X, C, Q)                                                                            \
    if (solo) crk_eval_kernel<X, C, true, Q><<<grid, b.evalThreads, 0, b.stream>>>(b.d_mem, bm, one);  \
    else crk_eval_kernel<X, C, false, Q><<<grid, b.evalThreads, 0, b.stream>>>(b.d_mem, bm, one)
    switch (v) {
      case 0: CRK_LAUNCH(false, false, false); break;
      case 1: CRK_LAUNCH(false, true, false); break;
      case 2: CRK_LAUNCH(true, false, false); break;
      case 3: CRK_LAUNCH(true, true, false); break;
      case 4: CRK_LAUNCH(false, false, true); break;
      case 5: CRK_LAUNCH(false, true, true); break;
      case 6: CRK_LAUNCH(true, false, true); break;
      default: CRK_LAUNCH(true, true, true); break;
    }
#undef CRK_LAUNCH
    batch_count_launch(b);
  }
  return cuda_status(cudaGetLastError(), "CRK evaluate");
}

}  // namespace sphgpu
