// CRKSPH derivatives, mixed-precision form.
//
// Same physics as CRKSPHHydroBase::evaluateDerivatives
// (src/CRKSPH/CRKSPHHydroBase.cc:646-1102) with CRKSPHKernelAndGradient
// (src/CRKSPH/CRKSPHUtilitiesInline.hh:58-129), pair arithmetic in FP32:
//   - relative position and velocity formed in FP64 and rounded once;
//   - table kernel, corrected kernel and gradient, Monaghan-Gingold Pi and
//     the pair force in FP32 (hardware rsqrt / reciprocal);
//   - per-node sums in FP32 with Kahan compensation;
//   - the moments and the correction-matrix inversion (crk.cu), volumes,
//     the per-node finish and everything outside the pair loop stay FP64.
// The 160-byte record keeps FP64 position and velocity and FP32 copies of
// the rest (m, rho, cs, P, det H, volume, H, A, B, grad A, grad B).
#include "problem.cuh"
#include "mixed.cuh"

namespace sphgpu {

namespace {

struct KahanF {
  float s, c;
  __device__ __forceinline__ void init() { s = 0.0f; c = 0.0f; }
  __device__ __forceinline__ void add(float x) {
    const float y = x - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
  }
  __device__ __forceinline__ double value() const { return (double)s - (double)c; }
};

struct F3 {
  float x, y, z;
};
__device__ __forceinline__ F3 symdotF(const float* h, const F3& r) {
  return F3{h[0]*r.x + h[1]*r.y + h[2]*r.z, h[1]*r.x + h[3]*r.y + h[4]*r.z, h[2]*r.x + h[4]*r.y + h[5]*r.z};
}
__device__ __forceinline__ float dotF(const F3& a, const F3& b) { return a.x*b.x + a.y*b.y + a.z*b.z; }

struct CMRec {
  double x, y, z, vx, vy, vz;
  float m, rho, cs, P, Hdet, vol, h[6], A, B[3], gA[3], gB[9];
};

__device__ __forceinline__ CMRec loadCMRec(const double* rec, int64_t k) {
  const double2* q = reinterpret_cast<const double2*>(rec + k*CMRECW);
  const double2 a0 = __ldg(q), a1 = __ldg(q + 1), a2 = __ldg(q + 2);
  const float4* f = reinterpret_cast<const float4*>(q + 3);
  const float4 f0 = __ldg(f), f1 = __ldg(f + 1), f2 = __ldg(f + 2), f3 = __ldg(f + 3);
  const float4 f4 = __ldg(f + 4), f5 = __ldg(f + 5), f6 = __ldg(f + 6);
  CMRec R;
  R.x = a0.x; R.y = a0.y; R.z = a1.x; R.vx = a1.y; R.vy = a2.x; R.vz = a2.y;
  R.m = f0.x; R.rho = f0.y; R.cs = f0.z; R.P = f0.w;
  R.Hdet = f1.x; R.vol = f1.y; R.h[0] = f1.z; R.h[1] = f1.w;
  R.h[2] = f2.x; R.h[3] = f2.y; R.h[4] = f2.z; R.h[5] = f2.w;
  R.A = f3.x; R.B[0] = f3.y; R.B[1] = f3.z; R.B[2] = f3.w;
  R.gA[0] = f4.x; R.gA[1] = f4.y; R.gA[2] = f4.z; R.gB[0] = f4.w;
  R.gB[1] = f5.x; R.gB[2] = f5.y; R.gB[3] = f5.z; R.gB[4] = f5.w;
  R.gB[5] = f6.x; R.gB[6] = f6.y; R.gB[7] = f6.z; R.gB[8] = f6.w;
  return R;
}

__global__ void __launch_bounds__(256) pack_crk_mixed_kernel(const Member* mem, BlockMap bm) {
  const MemberBlock mb = memberBlock(bm);
  const Member& MB = mem[mb.m];
  const int64_t n = MB.n;
  const int64_t k = mb.block*blockDim.x + threadIdx.x;
  if (k >= n + scalI(MB.scal, SC_G)) return;
  const double* S = MB.S;
  const double* K = MB.K;
  const int64_t r = k < n ? k : MB.groot[k - n];
  V3 x{S[S_X*n + r], S[S_Y*n + r], S[S_Z*n + r]};
  if (k >= n) x = ghostPosition(MB.prm.bcs, x, MB.gcode[k - n]);
  const Sym H{S[(S_H + 0)*n + r], S[(S_H + 1)*n + r], S[(S_H + 2)*n + r],
              S[(S_H + 3)*n + r], S[(S_H + 4)*n + r], S[(S_H + 5)*n + r]};
  double2* q = reinterpret_cast<double2*>(MB.mrec + k*CMRECW);
  q[0] = make_double2(x.x, x.y);
  q[1] = make_double2(x.z, S[S_VX*n + r]);
  q[2] = make_double2(S[S_VY*n + r], S[S_VZ*n + r]);
  float4* f = reinterpret_cast<float4*>(q + 3);
  auto kf = [&](int field) { return (float)K[(int64_t)field*n + r]; };
  f[0] = make_float4((float)S[S_M*n + r], (float)S[S_RHO*n + r], (float)S[S_CS*n + r], (float)S[S_P*n + r]);
  f[1] = make_float4((float)sdet(H), (float)S[S_VOL*n + r], (float)H.xx, (float)H.xy);
  f[2] = make_float4((float)H.xz, (float)H.yy, (float)H.yz, (float)H.zz);
  f[3] = make_float4(kf(K_A), kf(K_B), kf(K_B + 1), kf(K_B + 2));
  f[4] = make_float4(kf(K_GRADA), kf(K_GRADA + 1), kf(K_GRADA + 2), kf(K_GRADB));
  f[5] = make_float4(kf(K_GRADB + 1), kf(K_GRADB + 2), kf(K_GRADB + 3), kf(K_GRADB + 4));
  f[6] = make_float4(kf(K_GRADB + 5), kf(K_GRADB + 6), kf(K_GRADB + 7), kf(K_GRADB + 8));
}

__device__ __forceinline__ void tableF(const float* coef, int n, float invStep, float extent, float eta, float Hdet,
                                       float& W, float& gW) {
  if (eta < extent) {
    const float q = eta*invStep;
    int lb = (int)q;
    lb = lb < n - 1 ? lb : n - 1;
    const int i0 = lb < n - 3 ? lb : n - 3;
    const float x = q - (float)i0;
    const float2* c = reinterpret_cast<const float2*>(coef + 6*(i0 + 1));
    const float2 c01 = __ldg(c), c23 = __ldg(c + 1), c45 = __ldg(c + 2);
    W = Hdet*(c01.x + x*(c01.y + x*c23.x));
    gW = Hdet*(c23.y + x*(c45.x + x*c45.y));
  } else {
    W = 0.0f;
    gW = 0.0f;
  }
}

struct TabF {
  const float* coef;
  int n;
  float invStep, extent;
};

// |eta|, the unit vector of eta (x-axis for eta = 0) and the table values.
__device__ __forceinline__ void etaTable(const TabF& T, const F3& eta, float Hdet, float& W, float& gW, F3& u) {
  const float e2 = dotF(eta, eta);
  const float rinv = e2 > 0.0f ? __frsqrt_rn(e2) : 0.0f;
  u = e2 > 0.0f ? F3{eta.x*rinv, eta.y*rinv, eta.z*rinv} : F3{1.0f, 0.0f, 0.0f};
  tableF(T.coef, T.n, T.invStep, T.extent, e2*rinv, Hdet, W, gW);
}

// CRKSPHKernelAndGradient (LinearOrder) in FP32, node a's corrections.
__device__ __forceinline__ void crkKernelF(const F3& rij, float Wij, const F3& gradWij, float A, const float* B,
                                           const float* gA, const float* gB, float& WCRK, F3& gradWCRK) {
  const float Br = B[0]*rij.x + B[1]*rij.y + B[2]*rij.z;
  const float corr = A*(1.0f + Br);
  WCRK = corr*Wij;
  const float AW = A*Wij;
  const float gAW = (1.0f + Br)*Wij;
  gradWCRK.x = gradWij.x*corr + B[0]*AW + gA[0]*gAW + AW*(gB[0]*rij.x + gB[3]*rij.y + gB[6]*rij.z);
  gradWCRK.y = gradWij.y*corr + B[1]*AW + gA[1]*gAW + AW*(gB[1]*rij.x + gB[4]*rij.y + gB[7]*rij.z);
  gradWCRK.z = gradWij.z*corr + B[2]*AW + gA[2]*gAW + AW*(gB[2]*rij.x + gB[5]*rij.y + gB[8]*rij.z);
}

// CRKSPHMonaghanGingoldViscosity velocity reconstruction in FP32 (see
// crkQVelocityDifference in crk.cu): the cached velocity gradients projected
// on half the separation, van Leer limited, released near etaCrit.
__device__ __forceinline__ void loadQGradF(const double* qgrad, int64_t r, float* g) {
  const double2* q = reinterpret_cast<const double2*>(qgrad + r*QGRADW);
#pragma unroll
  for (int c = 0; c < 5; ++c) {
    const double2 v = __ldg(q + c);
    g[2*c] = (float)v.x;
    if (2*c + 1 < 9) g[2*c + 1] = (float)v.y;
  }
}

__device__ __forceinline__ F3 crkQVelocityDifferenceF(const Params& P, const double* qgrad, int64_t i, int64_t rj,
                                                      const F3& rij, const F3& vij, const F3& etai, const F3& etaj) {
  float gi[9], gj[9];
  loadQGradF(qgrad, i, gi);
  loadQGradF(qgrad, rj, gj);
  const F3 x{0.5f*rij.x, 0.5f*rij.y, 0.5f*rij.z};
  const F3 ti{gi[0]*x.x + gi[1]*x.y + gi[2]*x.z, gi[3]*x.x + gi[4]*x.y + gi[5]*x.z, gi[6]*x.x + gi[7]*x.y + gi[8]*x.z};
  const F3 tj{gj[0]*x.x + gj[1]*x.y + gj[2]*x.z, gj[3]*x.x + gj[4]*x.y + gj[5]*x.z, gj[6]*x.x + gj[7]*x.y + gj[8]*x.z};
  const float gradi = dotF(ti, x), gradj = dotF(tj, x);
  const float rI = gradi/(copysignf(1.0f, gradj)*fmaxf(1.0e-30f, fabsf(gradj)));
  const float rJ = gradj/(copysignf(1.0f, gradi)*fmaxf(1.0e-30f, fabsf(gradi)));
  const float r = fminf(rI, rJ);
  float phi = r > 0.0f ? 2.0f/(1.0f + r)*2.0f*r/(1.0f + r) : 0.0f;
  const float etaij = fminf(sqrtf(dotF(etai, etai)), sqrtf(dotF(etaj, etaj)));
  const float etaCrit = (float)P.etaCrit;
  if (etaij < etaCrit) {
    const float y = (etaij - etaCrit)/(float)P.etaFold;
    phi *= expf(-(y*y));
  }
  return F3{vij.x - phi*(ti.x + tj.x), vij.y - phi*(ti.y + tj.y), vij.z - phi*(ti.z + tj.z)};
}

template<bool XSPH, bool COMPAT, bool SOLO, bool QCRK>
__global__ void __launch_bounds__(128, 3) crk_eval_mixed_kernel(const Member* mem, BlockMap bm, const Member single) {
  const MemberBlock mb = memberBlock(bm);
  const Member& MB = SOLO ? single : mem[mb.m];   // one member: read from the kernel parameters
  const int64_t n = MB.n;
  const int64_t i = mb.block*blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Params& P = MB.prm;
  const double* rec = MB.mrec;
  const int64_t* offsets = MB.offsets;
  const int32_t* nbr = MB.nbr;
  double* D = MB.D;
  double* pacc = MB.pacc;
  const int64_t ecap = MB.ecap;
  const TabF T{MB.coefF, P.W.n, (float)(1.0/P.W.stepSize), (float)P.W.extent};
  const float eps2 = (float)P.eps2, Cl = (float)P.Cl, Cq = (float)P.Cq;
  const CMRec I = loadCMRec(rec, i);
  KahanF wns, effvp, viscW, DepsDt, DvDt[3], gradRho[3], XSPHdv[3], m2[6], DvDx[9];
  wns.init(); effvp.init(); viscW.init(); DepsDt.init();
#pragma unroll
  for (int c = 0; c < 3; ++c) { DvDt[c].init(); gradRho[c].init(); XSPHdv[c].init(); }
#pragma unroll
  for (int c = 0; c < 6; ++c) m2[c].init();
#pragma unroll
  for (int c = 0; c < 9; ++c) DvDx[c].init();
  float maxvp = 0.0f;
  const int64_t k0 = offsets[i], k1 = offsets[i + 1];
  for (int64_t k = k0; k < k1; ++k) {
    const int32_t j = __ldg(nbr + k);
    const CMRec J = loadCMRec(rec, j);
    const bool own = j > (int32_t)i;
    const F3 rij{(float)(I.x - J.x), (float)(I.y - J.y), (float)(I.z - J.z)};
    const F3 vij{(float)(I.vx - J.vx), (float)(I.vy - J.vy), (float)(I.vz - J.vz)};
    const F3 etai = symdotF(I.h, rij);
    const F3 etaj = symdotF(J.h, rij);
    float Wa, gWa, Wb, gWb;
    F3 ua, ub;
    etaTable(T, etai, I.Hdet, Wa, gWa, ua);
    etaTable(T, etaj, J.Hdet, Wb, gWb, ub);
    const F3 Hua = symdotF(I.h, ua), Hub = symdotF(J.h, ub);
    const float Wij = 0.5f*(Wa + Wb);
    const F3 gradWij{0.5f*(Hua.x*gWa + Hub.x*gWb), 0.5f*(Hua.y*gWa + Hub.y*gWb), 0.5f*(Hua.z*gWa + Hub.z*gWb)};
    const float gradWSPH = 0.5f*(gWa + gWb);
    // W^R_ij with i's corrections at r_ij, W^R_ji with j's at r_ji = -r_ij
    float Wj, Wi;
    F3 gradWj, gradWi;
    crkKernelF(rij, Wij, gradWij, I.A, I.B, I.gA, I.gB, Wj, gradWj);
    const F3 rji{-rij.x, -rij.y, -rij.z};
    const F3 gradWji{-gradWij.x, -gradWij.y, -gradWij.z};
    crkKernelF(rji, Wij, gradWji, J.A, J.B, J.gA, J.gB, Wi, gradWi);
    const F3 deltagrad{gradWj.x - gradWi.x, gradWj.y - gradWi.y, gradWj.z - gradWi.z};
    // SPH moments for the ideal H
    {
      const F3 gs{Hua.x*gWa, Hua.y*gWa, Hua.z*gWa};
      const float rij2 = dotF(rij, rij);
      const float r6 = rij2*rij2*rij2;
      const float thptS = r6 > 1.0e-30f ? __fdividef(1.0f, r6) : 1.0e30f;
      wns.add(fabsf(gradWSPH));
      const float g2 = dotF(gs, gs)*thptS;
      m2[0].add(rij.x*rij.x*g2); m2[1].add(rij.x*rij.y*g2); m2[2].add(rij.x*rij.z*g2);
      m2[3].add(rij.y*rij.y*g2); m2[4].add(rij.y*rij.z*g2); m2[5].add(rij.z*rij.z*g2);
    }
    // Monaghan-Gingold Pi (the CRKSPH Q sees the reconstructed velocities)
    F3 vQ = vij;
    if (QCRK) {
      const int64_t rootj = j < n ? (int64_t)j : (int64_t)__ldg(MB.groot + (j - n));
      vQ = crkQVelocityDifferenceF(P, MB.qgrad, i, rootj, rij, vij, etai, etaj);
    }
    const float mui = __fdividef(dotF(vQ, etai), dotF(etai, etai) + eps2);
    const float muj = __fdividef(dotF(vQ, etaj), dotF(etaj, etaj) + eps2);
    const float mi0 = fminf(0.0f, mui), mj0 = fminf(0.0f, muj);
    const float ei = -Cl*I.cs*(P.linearInExp ? mui : mi0) + Cq*(P.quadInExp ? -copysignf(1.0f, mui)*mui*mui : mi0*mi0);
    const float ej = -Cl*J.cs*(P.linearInExp ? muj : mj0) + Cq*(P.quadInExp ? -copysignf(1.0f, muj)*muj*muj : mj0*mj0);
    const float qsi = ei*I.rho, qsj = ej*J.rho;       // rho^2 * (e/rho)
    const float qsum = qsi + qsj;
    const float workQi = J.rho*ej*dotF(vij, deltagrad);
    const float Qi = I.rho*fabsf(ei);
    maxvp = fmaxf(maxvp, 4.0f*Qi);
    effvp.add(J.vol*Qi*Wj);
    const float f = 0.5f*I.vol*J.vol;
    const float invmi = __fdividef(1.0f, I.m);
    viscW.add(f*invmi*workQi);
    DvDx[0].add(-J.vol*vij.x*gradWj.x); DvDx[1].add(-J.vol*vij.x*gradWj.y); DvDx[2].add(-J.vol*vij.x*gradWj.z);
    DvDx[3].add(-J.vol*vij.y*gradWj.x); DvDx[4].add(-J.vol*vij.y*gradWj.y); DvDx[5].add(-J.vol*vij.y*gradWj.z);
    DvDx[6].add(-J.vol*vij.z*gradWj.x); DvDx[7].add(-J.vol*vij.z*gradWj.y); DvDx[8].add(-J.vol*vij.z*gradWj.z);
    const float drho = J.vol*(J.rho - I.rho);
    gradRho[0].add(gradWj.x*drho); gradRho[1].add(gradWj.y*drho); gradRho[2].add(gradWj.z*drho);
    const float Psum = I.P + J.P;
    const F3 force{(deltagrad.x*Psum + deltagrad.x*qsum)*f, (deltagrad.y*Psum + deltagrad.y*qsum)*f,
                   (deltagrad.z*Psum + deltagrad.z*qsum)*f};
    DvDt[0].add(-force.x*invmi); DvDt[1].add(-force.y*invmi); DvDt[2].add(-force.z*invmi);
    if (COMPAT) {
      // owner's pair acceleration (-force_owner/m_owner), FP32 in the mixed
      // form (both nodes of the pair read the same value)
      const double s = own ? -1.0/(double)I.m : 1.0/(double)J.m;
      float* pf = reinterpret_cast<float*>(pacc);
      pf[k] = (float)(s*(double)force.x);
      pf[ecap + k] = (float)(s*(double)force.y);
      pf[2*ecap + k] = (float)(s*(double)force.z);
    }
    DepsDt.add(f*(J.P*dotF(vij, deltagrad) + workQi)*invmi);
    if (XSPH) {
      const float w = J.vol*Wj;
      XSPHdv[0].add(-vij.x*w); XSPHdv[1].add(-vij.y*w); XSPHdv[2].add(-vij.z*w);
    }
  }
  // ---- per-node finish in FP64 (src/CRKSPH/CRKSPHHydroBase.cc:1036-1081)
  const double* S = MB.S;
  const Sym Hi{S[(S_H + 0)*n + i], S[(S_H + 1)*n + i], S[(S_H + 2)*n + i],
               S[(S_H + 3)*n + i], S[(S_H + 4)*n + i], S[(S_H + 5)*n + i]};
  const double rhoi = S[S_RHO*n + i], Hdeti = sdet(Hi);
  double dvdx[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) dvdx[c] = DvDx[c].value();
  const double tr = dvdx[0] + dvdx[4] + dvdx[8];
  const double DrhoDt = -rhoi*tr;
  double w = dmax(0.0, wns.value()/Hdeti);
  w = sgn(w)*pow(fabs(w), 0.3333333333333333);
  const V3 vi{S[S_VX*n + i], S[S_VY*n + i], S[S_VZ*n + i]};
  const V3 xdv{XSPHdv[0].value(), XSPHdv[1].value(), XSPHdv[2].value()};
  const V3 DxDt = XSPH ? vadd(vi, xdv) : vi;
  const Sym DHDt = smul(sdiv(sneg(Hi), 3.0), tr);
  double nPerhCur;
  if (fuzzyEqual(w, 0.0)) {
    nPerhCur = 0.5*P.nPerh;
  } else {
    nPerhCur = equivalentNodesPerSmoothingScale(P, w);
  }
  const double s = dmin(4.0, dmax(0.25, P.nPerh/(nPerhCur + 1.0e-30)));
  const double a = s < 1.0 ? 0.4*(1.0 + s*s) : 0.4*(1.0 + 1.0/(s*s*s));
  const double hi1 = dmin(P.hmax, dmax(P.hmin, (1.0/Hi.xx)*(1.0 - a + a*s)));
  const double hinv = 1.0/hi1;
  const double Hd2 = Hdeti*Hdeti;

  double* d = D + i;
  d[(D_DXDT + 0)*n] = DxDt.x; d[(D_DXDT + 1)*n] = DxDt.y; d[(D_DXDT + 2)*n] = DxDt.z;
  d[(D_DVDT + 0)*n] = DvDt[0].value(); d[(D_DVDT + 1)*n] = DvDt[1].value(); d[(D_DVDT + 2)*n] = DvDt[2].value();
  d[D_DRHODT*n] = DrhoDt;
  d[D_DEPSDT*n] = DepsDt.value();
  d[(D_DHDT + 0)*n] = DHDt.xx; d[(D_DHDT + 1)*n] = DHDt.xy; d[(D_DHDT + 2)*n] = DHDt.xz;
  d[(D_DHDT + 3)*n] = DHDt.yy; d[(D_DHDT + 4)*n] = DHDt.yz; d[(D_DHDT + 5)*n] = DHDt.zz;
  d[(D_HIDEAL + 0)*n] = hinv; d[(D_HIDEAL + 1)*n] = 0.0; d[(D_HIDEAL + 2)*n] = 0.0;
  d[(D_HIDEAL + 3)*n] = hinv; d[(D_HIDEAL + 4)*n] = 0.0; d[(D_HIDEAL + 5)*n] = hinv;
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    d[(D_DVDX + c)*n] = dvdx[c];
  }
  d[D_WNS*n] = w;
#pragma unroll
  for (int c = 0; c < 6; ++c) d[(D_M2 + c)*n] = m2[c].value()/Hd2;
  d[(D_XSPHDV + 0)*n] = xdv.x; d[(D_XSPHDV + 1)*n] = xdv.y; d[(D_XSPHDV + 2)*n] = xdv.z;
  d[D_MAXVP*n] = (double)maxvp;
  d[D_EFFVP*n] = effvp.value();
  d[D_VISCW*n] = viscW.value();
  double* K = MB.K;
  K[(K_GRADRHO + 0)*n + i] = gradRho[0].value();
  K[(K_GRADRHO + 1)*n + i] = gradRho[1].value();
  K[(K_GRADRHO + 2)*n + i] = gradRho[2].value();
}

bool isCrkMixed(const Problem& p) {
  return p.prm.hydro == SPHGPU_HYDRO_CRKSPH && p.cfg.precision == SPHGPU_PRECISION_MIXED;
}

}  // namespace

int launch_crk_eval_mixed(Batch& b) {
  BlockMap bm;
  unsigned grid = 0;
  SPH_TRY(batch_map_items(b, [&](const Problem& p) { return isCrkMixed(p) ? (b.capacityGrids ? p.candcap : p.n + p.G) : (int64_t)0; }, 256, &bm,
                          &grid));
  if (grid) { pack_crk_mixed_kernel<<<grid, 256, 0, b.stream>>>(b.d_mem, bm); batch_count_launch(b); }
  auto key = [](const Problem& p) {
    return (p.prm.qType == SPHGPU_Q_CRKSPH_MONAGHAN_GINGOLD ? 4 : 0) | (p.prm.XSPH ? 2 : 0) |
           (p.prm.compatible ? 1 : 0);
  };
  const bool solo = b.mem.size() == 1;
  const Member one = solo ? describe_member(*b.mem[0]) : Member{};
  bool present[8] = {false, false, false, false, false, false, false, false};
  for (Problem* p : b.mem) if (isCrkMixed(*p)) present[key(*p)] = true;
  for (int v = 0; v < 8; ++v) {
    if (!present[v]) continue;
    SPH_TRY(batch_map_items(b, [&](const Problem& p) { return isCrkMixed(p) && key(p) == v ? p.n : (int64_t)0; },
                            b.evalThreads, &bm, &grid));
    if (!grid) continue;
#define CRKM_LAUNCH(X, C, Q)                                                                                 \
    if (solo) crk_eval_mixed_kernel<X, C, true, Q><<<grid, b.evalThreads, 0, b.stream>>>(b.d_mem, bm, one);  \
    else crk_eval_mixed_kernel<X, C, false, Q><<<grid, b.evalThreads, 0, b.stream>>>(b.d_mem, bm, one)
    switch (v) {
      case 0: CRKM_LAUNCH(false, false, false); break;
      case 1: CRKM_LAUNCH(false, true, false); break;
      case 2: CRKM_LAUNCH(true, false, false); break;
      case 3: CRKM_LAUNCH(true, true, false); break;
      case 4: CRKM_LAUNCH(false, false, true); break;
      case 5: CRKM_LAUNCH(false, true, true); break;
      case 6: CRKM_LAUNCH(true, false, true); break;
      default: CRKM_LAUNCH(true, true, true); break;
    }
#undef CRKM_LAUNCH
    batch_count_launch(b);
  }
  return cuda_status(cudaGetLastError(), "CRK evaluate (mixed)");
}

}  // namespace sphgpu
