// SPH derivatives, mixed-precision form.
//
// Same physics as SPHHydroBase::evaluateDerivatives
// (src/SPH/SPHHydroBase.cc:471-928) with the pair arithmetic in FP32:
//   - relative position and velocity are formed in FP64 and rounded once;
//   - table kernel, gradient, Monaghan-Gingold Pi and pressure terms in FP32
//     (hardware rsqrt / reciprocal through __frsqrt_rn / __fdividef);
//   - per-node sums in FP32 with Kahan compensation;
//   - the per-node finish (3x3 M inverse, ideal H) and everything outside the
//     pair loop stay FP64.
// Pair terms are formed from node i's side (r_ij = r_i - r_j); every term of
// the reference is odd in r_ij and v_ij or even in both, so the i-side form
// equals the owner-side form up to rounding.  The stored pair accelerations
// are flipped to owner orientation for the compatible-energy update.
#include "problem.cuh"
#include "mixed.cuh"

namespace sphgpu {

namespace {

struct Kahan {
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

struct MRec {
  double x, y, z, vx, vy, vz;
  float m, rho, cs, Hdet, hxx, hxy, hxz, hyy, hyz, hzz, Prho, mrho, P, somega;
  float iso;           // 1: H = hxx I (the symmetric products reduce to scalings)
};

__device__ __forceinline__ MRec loadMRec(const double* mrec, int64_t k) {
  const double2* q = reinterpret_cast<const double2*>(mrec + k*MRECW);
  const double2 a0 = __ldg(q), a1 = __ldg(q + 1), a2 = __ldg(q + 2);
  const float4* f = reinterpret_cast<const float4*>(q + 3);
  const float4 b0 = __ldg(f), b1 = __ldg(f + 1), b2 = __ldg(f + 2), b3 = __ldg(f + 3);
  MRec R;
  R.x = a0.x; R.y = a0.y; R.z = a1.x; R.vx = a1.y; R.vy = a2.x; R.vz = a2.y;
  R.m = b0.x; R.rho = b0.y; R.cs = b0.z; R.Hdet = b0.w;
  R.hxx = b1.x; R.hxy = b1.y; R.hxz = b1.z; R.hyy = b1.w;
  R.hyz = b2.x; R.hzz = b2.y; R.Prho = b2.z; R.mrho = b2.w;
  R.P = b3.x; R.somega = b3.y; R.iso = b3.z;
  return R;
}

__global__ void table_to_float_kernel(const double* coef, int n, float* out) {
  for (int t = blockIdx.x*blockDim.x + threadIdx.x; t < 6*n; t += gridDim.x*blockDim.x) out[t] = (float)coef[t];
}

struct F3 {
  float x, y, z;
};
__device__ __forceinline__ F3 symdot(float xx, float xy, float xz, float yy, float yz, float zz, const F3& r) {
  return F3{xx*r.x + xy*r.y + xz*r.z, xy*r.x + yy*r.y + yz*r.z, xz*r.x + yz*r.y + zz*r.z};
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

// midInS0: the RK2 step's record-only mid point ran (update_kernel
// recordMid): the FP64 mid-point H and mass density of a member without
// grad-h are in S0, S holds the start of the step.
template<bool XSPH, bool TENSILE, bool COMPAT, bool SOLO, bool BALSARA>
__global__ void __launch_bounds__(128, SPH_MIXED_MIN_BLOCKS) sph_eval_mixed_kernel(const Member* mem, BlockMap bm, const Member single,
                                                                 int midInS0) {
  const MemberBlock mb = memberBlock(bm);
  const Member& MB = SOLO ? single : mem[mb.m];   // one member: read from the kernel parameters
  const int64_t n = MB.n;
  const int64_t i = mb.block*blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Params& P = MB.prm;
  const float* coefF = MB.coefF;
  const double* mrec = MB.mrec;
  const double* S = MB.S;
  const int64_t* offsets = MB.offsets;
  const int32_t* nbr = MB.nbr;
  double* D = MB.D;
  double* pacc = MB.pacc;
  const int64_t ecap = MB.ecap;
  const MRec I = loadMRec(mrec, i);
  const float invStep = (float)(1.0/P.W.stepSize), extent = (float)P.W.extent;
  const float eps2 = (float)P.eps2;
  const float Cl = (float)P.Cl, Cq = (float)P.Cq;
  Kahan rhoSum, norm, wns, effvp, viscW, DepsDt, XSPHw;
  Kahan DvDt[3], XSPHdv[3], m2[6], DvDx[9], M[9];
  rhoSum.init(); norm.init(); wns.init(); effvp.init(); viscW.init(); DepsDt.init(); XSPHw.init();
#pragma unroll
  for (int c = 0; c < 3; ++c) { DvDt[c].init(); XSPHdv[c].init(); }
#pragma unroll
  for (int c = 0; c < 6; ++c) m2[c].init();
#pragma unroll
  for (int c = 0; c < 9; ++c) { DvDx[c].init(); M[c].init(); }
  float maxvp = 0.0f;
  const float fsi = BALSARA ? (float)MB.fshear[i] : 1.0f;
  const int64_t k0 = offsets[i], k1 = offsets[i + 1];
  for (int64_t k = k0; k < k1; ++k) {
    const int32_t j = __ldg(nbr + k);
    const MRec J = loadMRec(mrec, j);
    // the Balsara shear correction of the pair (max of the two nodes'), else 1
    const float fs = BALSARA ? fmaxf(fsi, (float)MB.fshear[j < n ? (int64_t)j : (int64_t)MB.groot[j - n]]) : 1.0f;
    const float ClP = Cl*fs, CqP = Cq*fs;
    // FP64 differences, rounded once
    const F3 rij{(float)(I.x - J.x), (float)(I.y - J.y), (float)(I.z - J.z)};
    const F3 vij{(float)(I.vx - J.vx), (float)(I.vy - J.vy), (float)(I.vz - J.vz)};
    // isotropic H (the common case): H r = hxx r, bit-identical to the full product
    const bool isoPair = I.iso != 0.0f && J.iso != 0.0f;
    F3 etai, etaj;
    if (isoPair) {
      etai = F3{I.hxx*rij.x, I.hxx*rij.y, I.hxx*rij.z};
      etaj = F3{J.hxx*rij.x, J.hxx*rij.y, J.hxx*rij.z};
    } else {
      etai = symdot(I.hxx, I.hxy, I.hxz, I.hyy, I.hyz, I.hzz, rij);
      etaj = symdot(J.hxx, J.hxy, J.hxz, J.hyy, J.hyz, J.hzz, rij);
    }
    const float e2i = etai.x*etai.x + etai.y*etai.y + etai.z*etai.z;
    const float e2j = etaj.x*etaj.x + etaj.y*etaj.y + etaj.z*etaj.z;
    const float rinvi = e2i > 0.0f ? __frsqrt_rn(e2i) : 0.0f;
    const float rinvj = e2j > 0.0f ? __frsqrt_rn(e2j) : 0.0f;
    const float etaMagi = e2i*rinvi, etaMagj = e2j*rinvj;
    const F3 ui = e2i > 0.0f ? F3{etai.x*rinvi, etai.y*rinvi, etai.z*rinvi} : F3{1.0f, 0.0f, 0.0f};
    const F3 uj = e2j > 0.0f ? F3{etaj.x*rinvj, etaj.y*rinvj, etaj.z*rinvj} : F3{1.0f, 0.0f, 0.0f};
    F3 Hetai, Hetaj;
    if (isoPair) {
      Hetai = F3{I.hxx*ui.x, I.hxx*ui.y, I.hxx*ui.z};
      Hetaj = F3{J.hxx*uj.x, J.hxx*uj.y, J.hxx*uj.z};
    } else {
      Hetai = symdot(I.hxx, I.hxy, I.hxz, I.hyy, I.hyz, I.hzz, ui);
      Hetaj = symdot(J.hxx, J.hxy, J.hxz, J.hyy, J.hyz, J.hzz, uj);
    }
    float Wi, gWi, Wj, gWj;
    tableF(coefF, P.W.n, invStep, extent, etaMagi, I.Hdet, Wi, gWi);
    tableF(coefF, P.W.n, invStep, extent, etaMagj, J.Hdet, Wj, gWj);
    const F3 gradWi{Hetai.x*gWi, Hetai.y*gWi, Hetai.z*gWi};
    const F3 gradWj{Hetaj.x*gWj, Hetaj.y*gWj, Hetaj.z*gWj};

    const float rij2 = rij.x*rij.x + rij.y*rij.y + rij.z*rij.z;
    const float r6 = rij2*rij2*rij2;
    const float thptS = r6 > 1.0e-30f ? __fdividef(1.0f, r6) : 1.0e30f;
    wns.add(fabsf(gWi));
    const float g2 = (gradWi.x*gradWi.x + gradWi.y*gradWi.y + gradWi.z*gradWi.z)*thptS;
    m2[0].add(rij.x*rij.x*g2); m2[1].add(rij.x*rij.y*g2); m2[2].add(rij.x*rij.z*g2);
    m2[3].add(rij.y*rij.y*g2); m2[4].add(rij.y*rij.z*g2); m2[5].add(rij.z*rij.z*g2);
    rhoSum.add(J.m*Wi);
    norm.add(I.mrho*Wi);

    // Monaghan-Gingold Pi
    const float mui = __fdividef(vij.x*etai.x + vij.y*etai.y + vij.z*etai.z, e2i + eps2);
    const float muj = __fdividef(vij.x*etaj.x + vij.y*etaj.y + vij.z*etaj.z, e2j + eps2);
    const float mi0 = fminf(0.0f, mui), mj0 = fminf(0.0f, muj);
    const float ei = -ClP*I.cs*(P.linearInExp ? mui : mi0) + CqP*(P.quadInExp ? -copysignf(1.0f, mui)*mui*mui : mi0*mi0);
    const float ej = -ClP*J.cs*(P.linearInExp ? muj : mj0) + CqP*(P.quadInExp ? -copysignf(1.0f, muj)*muj*muj : mj0*mj0);
    const float qi = __fdividef(ei, I.rho), qj = __fdividef(ej, J.rho);
    const F3 Qacci{0.5f*qi*gradWi.x, 0.5f*qi*gradWi.y, 0.5f*qi*gradWi.z};
    const F3 Qaccj{0.5f*qj*gradWj.x, 0.5f*qj*gradWj.y, 0.5f*qj*gradWj.z};
    const float workQi = vij.x*Qacci.x + vij.y*Qacci.y + vij.z*Qacci.z;
    const float Qi = I.rho*I.rho*fabsf(qi);
    maxvp = fmaxf(maxvp, Qi);
    effvp.add(J.mrho*Qi*Wi);
    viscW.add(J.m*workQi);

    float Prhoi = I.Prho, Prhoj = J.Prho;
    if (TENSILE) {
      const bool own = j > (int32_t)i;
      const float Wo = own ? Wi : Wj, Hdo = own ? I.Hdet : J.Hdet;
      const float x = __fdividef(Wo, Hdo*(float)P.WnPerh);
      const float fij = (float)P.epsTensile*(x*x*x*x);
      Prhoi = __fdividef(I.somega*(I.P + fij*(I.P < 0.0f ? -I.P : 0.0f)), I.rho*I.rho);
      Prhoj = __fdividef(J.somega*(J.P + fij*(J.P < 0.0f ? -J.P : 0.0f)), J.rho*J.rho);
    }
    const F3 dd{Prhoi*gradWi.x + Prhoj*gradWj.x + Qacci.x + Qaccj.x,
                Prhoi*gradWi.y + Prhoj*gradWj.y + Qacci.y + Qaccj.y,
                Prhoi*gradWi.z + Prhoj*gradWj.z + Qacci.z + Qaccj.z};
    DvDt[0].add(-J.m*dd.x); DvDt[1].add(-J.m*dd.y); DvDt[2].add(-J.m*dd.z);
    DepsDt.add(J.m*(Prhoi*(vij.x*gradWi.x + vij.y*gradWi.y + vij.z*gradWi.z) + workQi));
    if (COMPAT) {
      // the owner's pair acceleration: -m_other*deltaDvDt in owner orientation
      // (FP32 in the mixed form; both nodes of the pair read the same value)
      const bool own = j > (int32_t)i;
      const float s = own ? -J.m : I.m;
      float* pf = reinterpret_cast<float*>(pacc);
      pf[k] = s*dd.x;
      pf[ecap + k] = s*dd.y;
      pf[2*ecap + k] = s*dd.z;
    }
    const float mj = J.m;
    const F3 mg{mj*gradWi.x, mj*gradWi.y, mj*gradWi.z};
    DvDx[0].add(-vij.x*mg.x); DvDx[1].add(-vij.x*mg.y); DvDx[2].add(-vij.x*mg.z);
    DvDx[3].add(-vij.y*mg.x); DvDx[4].add(-vij.y*mg.y); DvDx[5].add(-vij.y*mg.z);
    DvDx[6].add(-vij.z*mg.x); DvDx[7].add(-vij.z*mg.y); DvDx[8].add(-vij.z*mg.z);
    M[0].add(-rij.x*mg.x); M[1].add(-rij.x*mg.y); M[2].add(-rij.x*mg.z);
    M[3].add(-rij.y*mg.x); M[4].add(-rij.y*mg.y); M[5].add(-rij.y*mg.z);
    M[6].add(-rij.z*mg.x); M[7].add(-rij.z*mg.y); M[8].add(-rij.z*mg.z);
    if (XSPH) {
      const float w = 0.5f*(I.mrho*Wi + J.mrho*Wj);
      XSPHw.add(w);
      XSPHdv[0].add(-w*vij.x); XSPHdv[1].add(-w*vij.y); XSPHdv[2].add(-w*vij.z);
    }
  }

  // ---- per-node finish in FP64 (src/SPH/SPHHydroBase.cc:834-902)
  // exact FP64 node values for the finish
  const double* Sm = midInS0 && !P.gradh && !P.balsara ? MB.S0 : S;
  const Sym Hi{Sm[(S_H + 0)*n + i], Sm[(S_H + 1)*n + i], Sm[(S_H + 2)*n + i],
               Sm[(S_H + 3)*n + i], Sm[(S_H + 4)*n + i], Sm[(S_H + 5)*n + i]};
  const double mi = S[S_M*n + i], rhoi = Sm[S_RHO*n + i], Hdeti = sdet(Hi);
  const int numNeighbors = (int)(k1 - k0);
  double rhoS = rhoSum.value() + mi*P.W0*Hdeti;
  double nrm = norm.value() + mi/rhoi*P.W0*Hdeti;
  T9 Mi{M[0].value(), M[1].value(), M[2].value(), M[3].value(), M[4].value(), M[5].value(),
        M[6].value(), M[7].value(), M[8].value()};
  T9 DvDxi{DvDx[0].value(), DvDx[1].value(), DvDx[2].value(), DvDx[3].value(), DvDx[4].value(),
           DvDx[5].value(), DvDx[6].value(), DvDx[7].value(), DvDx[8].value()};
  if (P.correctVelGrad && fabs(tdet(Mi)) > 1.0e-10 && numNeighbors > 8) {
    Mi = tinverse(Mi);
    DvDxi = tdot(DvDxi, Mi);
  } else {
    DvDxi = tdiv(DvDxi, rhoi);
  }
  const double DrhoDt = -rhoi*ttrace(DvDxi);
  double w = dmax(0.0, wns.value()/Hdeti);
  w = cbrt(w);
  Sym m2s{m2[0].value(), m2[1].value(), m2[2].value(), m2[3].value(), m2[4].value(), m2[5].value()};
  m2s = sdiv(m2s, Hdeti*Hdeti);
  const V3 vi{I.vx, I.vy, I.vz};
  V3 DxDt = vi;
  double xw = XSPHw.value();
  V3 xdv{XSPHdv[0].value(), XSPHdv[1].value(), XSPHdv[2].value()};
  if (XSPH) {
    xw += Hdeti*mi/rhoi*P.W0;
    DxDt = vadd(vi, vdiv(xdv, dmax(1.0e-30, xw)));
  }
  const Sym DHDt = smul(sdiv(sneg(Hi), 3.0), ttrace(DvDxi));
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

  double* d = D + i;
  d[(D_DXDT + 0)*n] = DxDt.x; d[(D_DXDT + 1)*n] = DxDt.y; d[(D_DXDT + 2)*n] = DxDt.z;
  d[(D_DVDT + 0)*n] = DvDt[0].value(); d[(D_DVDT + 1)*n] = DvDt[1].value(); d[(D_DVDT + 2)*n] = DvDt[2].value();
  d[D_DRHODT*n] = DrhoDt;
  d[D_DEPSDT*n] = DepsDt.value();
  d[(D_DHDT + 0)*n] = DHDt.xx; d[(D_DHDT + 1)*n] = DHDt.xy; d[(D_DHDT + 2)*n] = DHDt.xz;
  d[(D_DHDT + 3)*n] = DHDt.yy; d[(D_DHDT + 4)*n] = DHDt.yz; d[(D_DHDT + 5)*n] = DHDt.zz;
  d[(D_HIDEAL + 0)*n] = hinv; d[(D_HIDEAL + 1)*n] = 0.0; d[(D_HIDEAL + 2)*n] = 0.0;
  d[(D_HIDEAL + 3)*n] = hinv; d[(D_HIDEAL + 4)*n] = 0.0; d[(D_HIDEAL + 5)*n] = hinv;
  const double* dv = &DvDxi.xx;
  const double* mm = &Mi.xx;
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    d[(D_DVDX + c)*n] = dv[c];
    d[(D_M + c)*n] = mm[c];
  }
  d[D_RHOSUM*n] = rhoS;
  d[D_NORM*n] = nrm;
  d[D_WNS*n] = w;
  d[(D_M2 + 0)*n] = m2s.xx; d[(D_M2 + 1)*n] = m2s.xy; d[(D_M2 + 2)*n] = m2s.xz;
  d[(D_M2 + 3)*n] = m2s.yy; d[(D_M2 + 4)*n] = m2s.yz; d[(D_M2 + 5)*n] = m2s.zz;
  d[D_XSPHW*n] = xw;
  d[(D_XSPHDV + 0)*n] = xdv.x; d[(D_XSPHDV + 1)*n] = xdv.y; d[(D_XSPHDV + 2)*n] = xdv.z;
  d[D_MAXVP*n] = (double)maxvp;
  d[D_EFFVP*n] = effvp.value();
  d[D_VISCW*n] = viscW.value();
}

}  // namespace

int prepare_mixed(Batch& b) {
  for (Problem* pp : b.mem) {
    Problem& p = *pp;
    if (p.cfg.precision != SPHGPU_PRECISION_MIXED) continue;
    if (p.coefF == nullptr) {
      if (dev_alloc(reinterpret_cast<void**>(&p.coefF), sizeof(float)*6*(size_t)p.prm.W.n) != cudaSuccess) {
        set_error("mixed table allocation failed");
        return SPHGPU_ERR_NOMEM;
      }
      table_to_float_kernel<<<8, 256, 0, b.stream>>>(p.prm.W.coef, p.prm.W.n, p.coefF); ++p.launches;
      b.memDirty = true;
    }
    const int64_t need = p.candcap;
    if (need > p.mreccap) {
      cudaStreamSynchronize(b.stream);
      dev_free(p.mrec);
      p.mrec = nullptr;
      if (dev_alloc(reinterpret_cast<void**>(&p.mrec), sizeof(double)*(p.prm.hydro == SPHGPU_HYDRO_CRKSPH ? CMRECW : MRECW)*(size_t)need) != cudaSuccess) {
        p.mreccap = 0;
        set_error("mixed record allocation failed");
        return SPHGPU_ERR_NOMEM;
      }
      p.mreccap = need;
      b.memDirty = true;
    }
  }
  if (b.memDirty) SPH_TRY(batch_upload(b));
  return SPHGPU_OK;
}

// SPH members in the mixed form (CRKSPH members in the mixed form have their
// own records and kernels, crk_mixed.cu)
bool mixedSph(const Problem& p) {
  return p.cfg.precision == SPHGPU_PRECISION_MIXED && p.prm.hydro == SPHGPU_HYDRO_SPH;
}

// One launch of the mixed pair kernel variant <XSPH, TENSILE, COMPAT, BALSARA>.
template<bool X, bool T, bool C, bool B>
void launch_mixed_variant(Batch& b, unsigned grid, BlockMap bm, const Member& one, bool solo, int mid) {
  if (solo) sph_eval_mixed_kernel<X, T, C, true, B><<<grid, b.evalThreads, 0, b.stream>>>(b.d_mem, bm, one, mid);
  else sph_eval_mixed_kernel<X, T, C, false, B><<<grid, b.evalThreads, 0, b.stream>>>(b.d_mem, bm, one, mid);
}
using MixedLaunch = void (*)(Batch&, unsigned, BlockMap, const Member&, bool, int);
// indexed by BALSARA << 3 | XSPH << 2 | TENSILE << 1 | COMPAT
const MixedLaunch kMixedLaunch[16] = {
    &launch_mixed_variant<false, false, false, false>, &launch_mixed_variant<false, false, true, false>,
    &launch_mixed_variant<false, true, false, false>, &launch_mixed_variant<false, true, true, false>,
    &launch_mixed_variant<true, false, false, false>, &launch_mixed_variant<true, false, true, false>,
    &launch_mixed_variant<true, true, false, false>, &launch_mixed_variant<true, true, true, false>,
    &launch_mixed_variant<false, false, false, true>, &launch_mixed_variant<false, false, true, true>,
    &launch_mixed_variant<false, true, false, true>, &launch_mixed_variant<false, true, true, true>,
    &launch_mixed_variant<true, false, false, true>, &launch_mixed_variant<true, false, true, true>,
    &launch_mixed_variant<true, true, false, true>, &launch_mixed_variant<true, true, true, true>};

int launch_eval_sph_mixed(Batch& b) {
  auto mixed = mixedSph;
  SPH_TRY(pack_mixed(b, false));
  auto key = [](const Problem& p) {
    return (p.prm.balsara ? 8 : 0) | (p.prm.XSPH ? 4 : 0) | (p.prm.epsTensile != 0.0 ? 2 : 0) |
           (p.prm.compatible ? 1 : 0);
  };
  const bool solo = b.mem.size() == 1;
  const Member one = solo ? describe_member(*b.mem[0]) : Member{};
  const int mid = b.midInS0 ? 1 : 0;
  bool present[16] = {};
  for (Problem* p : b.mem) if (mixed(*p)) present[key(*p)] = true;
  for (int v = 0; v < 16; ++v) {
    if (!present[v]) continue;
    BlockMap bm;
    unsigned grid = 0;
    SPH_TRY(batch_map_items(b, [&](const Problem& p) { return mixed(p) && key(p) == v ? p.n : (int64_t)0; }, b.evalThreads,
                            &bm, &grid));
    if (!grid) continue;
    kMixedLaunch[v](b, grid, bm, one, solo, mid);
    batch_count_launch(b);
  }
  return cuda_status(cudaGetLastError(), "evaluate (mixed)");
}

}  // namespace sphgpu
