// SPH hydro kernels, plain FP64 form (compiled with -fmad=false).
//
// Replaces the reference's serial loops:
//   pack_records         Integrator::applyGhostBoundaries (src/Integrator/Integrator.cc:602-660)
//   sph_eval_fp64        SPHHydroBase::evaluateDerivatives (src/SPH/SPHHydroBase.cc:471-928)
//   gradh                computeSPHOmegaGradhCorrection (src/SPH/computeSPHOmegaGradhCorrection.cc:28-137)
//   sum_density          computeSPHSumMassDensity (src/SPH/computeSPHSumMassDensity.cc:27-111)
//   compatible_energy    SpecificThermalEnergyPolicy::update (src/Hydro/SpecificThermalEnergyPolicy.cc:66-189)
//   update               State::update with the SPH policies (src/DataBase/State.cc:166-287,
//                        IncrementFieldList.cc:107-151, IncrementBoundedState.cc:120-136,
//                        ReplaceBoundedState.cc:121-150, PressurePolicy/SoundSpeedPolicy)
//   hydro_dt             GenericHydro::dt (src/Physics/GenericHydro.cc:114-331)
//   enforce_boundaries   PeriodicBoundary violation mapping (src/Boundary/PeriodicBoundary.cc:145-203)
//
// Pair loops gather: one thread owns node i and walks its ascending CSR row.
// The reference visits each unordered pair once, from the lower index (the
// "owner"), and scatters to both nodes.  Here every pair term is formed in
// owner orientation (r_ij = r_owner - r_other, owner-side Q, owner-side
// tensile factor) and only node i's side is accumulated.  Node i's sums then
// receive the same terms in the same order as in the reference: first the
// pairs owned by lower indices (ascending), then its own (ascending, ghosts
// last), with self terms inserted where the reference adds them.
#include <cfloat>

#include "problem.cuh"

namespace sphgpu {

namespace {

constexpr double kFltMin = 1.17549435082228750797e-38;   // FLT_MIN
constexpr double kFltMax = 3.40282346638528859812e+38;   // FLT_MAX
constexpr double kDblEps = 2.220446049250313e-16;

constexpr int kConsBlocks = 148*4;   // conservation partial sums per member

__device__ __forceinline__ double ldg(const double* p) { return __ldg(p); }

struct Rec {
  V3 r, v;
  double m, rho, cs, Hdet;
  Sym H;
  double Prho, mrho, P, somega;
};

__device__ __forceinline__ Rec loadRec(const double* rec, int64_t k) {
  const double2* q = reinterpret_cast<const double2*>(rec + k*RECW);
  const double2 a0 = __ldg(q + 0), a1 = __ldg(q + 1), a2 = __ldg(q + 2), a3 = __ldg(q + 3), a4 = __ldg(q + 4);
  const double2 a5 = __ldg(q + 5), a6 = __ldg(q + 6), a7 = __ldg(q + 7), a8 = __ldg(q + 8), a9 = __ldg(q + 9);
  Rec R;
  // the layout of writeRecord (problem.cuh)
  R.r = V3{a0.x, a0.y, a1.x};
  R.m = a1.y; R.Hdet = a2.x;
  R.H = Sym{a2.y, a3.x, a3.y, a4.x, a4.y, a5.x};
  R.v = V3{a5.y, a6.x, a6.y};
  R.rho = a7.x; R.cs = a7.y;
  R.Prho = a8.x; R.mrho = a8.y; R.P = a9.x; R.somega = a9.y;
  return R;
}

__device__ __forceinline__ V3 selv(bool c, const V3& a, const V3& b) {
  return V3{c ? a.x : b.x, c ? a.y : b.y, c ? a.z : b.z};
}
__device__ __forceinline__ Sym sels(bool c, const Sym& a, const Sym& b) {
  return Sym{c ? a.xx : b.xx, c ? a.xy : b.xy, c ? a.xz : b.xz, c ? a.yy : b.yy, c ? a.yz : b.yz, c ? a.zz : b.zz};
}

// ---------------------------------------------------------------- records
// Pair records of the nodes [first, n + G): every node, or only the ghosts
// when the update kernel has already packed the internal nodes.  A ghost's
// record is its root's with the position mapped through the periodic planes.
__device__ __forceinline__ void nodeRecordState(const Member& M, int64_t k, V3& x, V3& v, double& m, double& rho,
                                                double& cs, double& P, double& omega, Sym& H) {
  const double* S = M.S;
  const int64_t n = M.n;
  const int64_t r = k < n ? k : M.groot[k - n];
  x = V3{S[S_X*n + r], S[S_Y*n + r], S[S_Z*n + r]};
  if (k >= n) x = ghostPosition(M.prm.bcs, x, M.gcode[k - n]);
  v = V3{S[S_VX*n + r], S[S_VY*n + r], S[S_VZ*n + r]};
  H = Sym{S[(S_H + 0)*n + r], S[(S_H + 1)*n + r], S[(S_H + 2)*n + r],
          S[(S_H + 3)*n + r], S[(S_H + 4)*n + r], S[(S_H + 5)*n + r]};
  m = S[S_M*n + r]; rho = S[S_RHO*n + r]; cs = S[S_CS*n + r]; P = S[S_P*n + r]; omega = S[S_OMEGA*n + r];
}

// A ghost's record from its root's record (written by the update kernel):
// every field but the position is the root's, the position is mapped
// through the periodic planes, so the record equals the one packed from the
// root's state.  W doubles per record, position in the first three.
template<int W>
__device__ __forceinline__ void ghostFromRoot(const Member& M, double* recs, int64_t k) {
  const int64_t r = M.groot[k - M.n];
  const double2* src = reinterpret_cast<const double2*>(recs + r*W);
  double2* dst = reinterpret_cast<double2*>(recs + k*W);
  const double2 p01 = src[0], p2v = src[1];
  const V3 x = ghostPosition(M.prm.bcs, V3{p01.x, p01.y, p2v.x}, M.gcode[k - M.n]);
  dst[0] = make_double2(x.x, x.y);
  dst[1] = make_double2(x.z, p2v.y);
#pragma unroll
  for (int c = 2; c < W/2; ++c) dst[c] = src[c];
}

// ghostsOnly: the update kernel wrote the internal nodes' records (in the
// RK2 step the state may then hold the start of the step, not the records'
// mid point), so the ghosts copy their roots' records.
__global__ void __launch_bounds__(256) pack_records_kernel(const Member* mem, BlockMap bm, int ghostsOnly) {
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const int64_t k = (ghostsOnly ? M.n : 0) + mb.block*blockDim.x + threadIdx.x;
  if (k >= M.n + scalI(M.scal, SC_G)) return;
  if (ghostsOnly) { ghostFromRoot<RECW>(M, M.rec, k); return; }
  V3 x, v; double m, rho, cs, P, omega; Sym H;
  nodeRecordState(M, k, x, v, m, rho, cs, P, omega, H);
  writeRecord(M.rec, k, x, v, m, rho, cs, P, omega, H);
}

__global__ void __launch_bounds__(256) pack_mixed_kernel(const Member* mem, BlockMap bm, int ghostsOnly) {
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const int64_t k = (ghostsOnly ? M.n : 0) + mb.block*blockDim.x + threadIdx.x;
  if (k >= M.n + scalI(M.scal, SC_G)) return;
  if (ghostsOnly) { ghostFromRoot<MRECW>(M, M.mrec, k); return; }
  V3 x, v; double m, rho, cs, P, omega; Sym H;
  nodeRecordState(M, k, x, v, m, rho, cs, P, omega, H);
  writeMixedRecord(M.mrec, k, x, v, m, rho, cs, P, omega, H);
}

// ---------------------------------------------------------------- derivatives
// The terms of one directed pair (i, j) that node i's sums take, formed in
// owner orientation (own: i owns the pair, j > i).  The reference forms every
// pair term from the owner A and the other node B.  Here each quantity is
// formed once for node i and once for node j, with the same operands in the
// same order: with the owner-oriented separation r_ij = r_A - r_B (= r_i -
// r_j or its exact negation), eta_i = H_i r_ij is eta_A when i owns the pair
// and eta_B otherwise, and likewise for j.  Sums of two pair terms are
// commutative and keep their bits; where three or more are added the owner's
// order is selected explicitly.
struct PairTerms {
  V3 rij, vij, gradWI, dd;      // dd: deltaDvDt
  double WI, WJ, gWI, thptS, QI, workQI, PrhoI, mj, mrhoj;
  bool own;
};

template<bool TENSILE>
__device__ __forceinline__ PairTerms pairTerms(const Rec& I, bool isoI, const Rec& J, bool own, const Params& P,
                                               double Cl, double Cq) {
  PairTerms t;
  t.own = own;
  t.mj = J.m;
  t.mrhoj = J.mrho;
  const V3 d = vsub(I.r, J.r);
  const V3 rij = own ? d : V3{-d.x, -d.y, -d.z};
  const V3 dv = vsub(I.v, J.v);
  const V3 vij = own ? dv : V3{-dv.x, -dv.y, -dv.z};
  t.rij = rij;
  t.vij = vij;
  // H = h I (the common case): every H product reduces to a scaling with
  // the same bits (the off-diagonal terms add exact zeros)
  const bool iso = isoI && isoSym(J.H);
  const V3 etaI = iso ? vmul(rij, I.H.xx) : sdot(I.H, rij);
  const V3 etaJ = iso ? vmul(rij, J.H.xx) : sdot(J.H, rij);
  const V3 uI = unitVector(etaI), uJ = unitVector(etaJ);
  const V3 HetaI = iso ? vmul(uI, I.H.xx) : sdot(I.H, uI);
  const V3 HetaJ = iso ? vmul(uJ, J.H.xx) : sdot(J.H, uJ);
  double WI, gWI, WJ, gWJ;
  tableKernelAndGrad(P.W, mag(etaI), I.Hdet, WI, gWI);
  tableKernelAndGrad(P.W, mag(etaJ), J.Hdet, WJ, gWJ);
  const V3 gradWI = vmul(HetaI, gWI);    // node i's side of the pair
  const V3 gradWJ = vmul(HetaJ, gWJ);
  t.WI = WI; t.WJ = WJ; t.gWI = gWI; t.gradWI = gradWI;
  // moments for the ideal H
  const double rij2 = mag2(rij);
  t.thptS = safeInvVar(rij2*rij2*rij2);
  // Monaghan-Gingold Pi_ij
  const double muI = dot(vij, etaI)/(mag2(etaI) + P.eps2);
  const double muJ = dot(vij, etaJ)/(mag2(etaJ) + P.eps2);
  const double mI0 = dmin(0.0, muI), mJ0 = dmin(0.0, muJ);
  const double eI = -Cl*I.cs*(P.linearInExp ? muI : mI0) + Cq*(P.quadInExp ? -sgn(muI)*muI*muI : mI0*mI0);
  const double eJ = -Cl*J.cs*(P.linearInExp ? muJ : mJ0) + Cq*(P.quadInExp ? -sgn(muJ)*muJ*muJ : mJ0*mJ0);
  const double qI = eI/I.rho, qJ = eJ/J.rho;   // (e/rho) * Tensor::one
  // 0.5*(Pi * gradWQ), with WQ = W (same table): the off-diagonal zeros of
  // Pi only add signed zeros.
  const V3 QaccI = vmul(vmul(gradWI, qI), 0.5);
  const V3 QaccJ = vmul(vmul(gradWJ, qJ), 0.5);
  t.workQI = dot(vij, QaccI);
  t.QI = I.rho*I.rho*fabs(qI);
  // pressure terms (tensile correction uses the owner's W)
  double PrhoI, PrhoJ;
  if (TENSILE) {
    const double x = own ? WI/(I.Hdet*P.WnPerh) : WJ/(J.Hdet*P.WnPerh);
    const double fij = P.epsTensile*(x*x*x*x);
    const double RI = fij*(I.P < 0.0 ? -I.P : 0.0);
    const double RJ = fij*(J.P < 0.0 ? -J.P : 0.0);
    PrhoI = I.somega*(I.P + RI)/(I.rho*I.rho);
    PrhoJ = J.somega*(J.P + RJ)/(J.rho*J.rho);
  } else {
    PrhoI = I.Prho;
    PrhoJ = J.Prho;
  }
  t.PrhoI = PrhoI;
  // ((gradW_A P_A + gradW_B P_B) + Qacc_A) + Qacc_B
  const V3 pp = vadd(vmul(gradWI, PrhoI), vmul(gradWJ, PrhoJ));
  t.dd = vadd(vadd(pp, own ? QaccI : QaccJ), own ? QaccJ : QaccI);
  return t;
}

// SPHHydroBase::evaluateDerivatives: one thread per internal node i, its CSR
// row in ascending order (the reference's accumulation order), node i's side
// of every pair.
template<bool XSPH, bool TENSILE, bool COMPAT, bool SOLO, bool BALSARA>
__global__ void __launch_bounds__(128, SPH_FP64_MIN_BLOCKS) sph_eval_fp64_kernel(const Member* mem, BlockMap bm, const Member single) {
  const MemberBlock mb = memberBlock(bm);
  const Member& MB = SOLO ? single : mem[mb.m];   // one member: read from the kernel parameters
  const int64_t n = MB.n;
  const int64_t i = mb.block*blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Params& P = MB.prm;
  const double* rec = MB.rec;
  const int64_t* offsets = MB.offsets;
  const int32_t* nbr = MB.nbr;
  double* D = MB.D;
  double* pacc = MB.pacc;
  const int64_t ecap = MB.ecap;
#if SPH_FP64_SHARED_I
  // node i's record lives in shared memory: the pair loop reads its fields
  // from there instead of holding 19 doubles in registers across the loop
  __shared__ Rec sI[128];
  sI[threadIdx.x] = loadRec(rec, i);
  const Rec& I = sI[threadIdx.x];
#else
  const Rec I = loadRec(rec, i);
#endif
  const bool isoI = isoSym(I.H);
  double rhoSum = 0.0, norm = 0.0, wns = 0.0, maxvp = 0.0, effvp = 0.0, viscW = 0.0, DepsDt = 0.0;
  double XSPHw = 0.0;
  V3 DvDt{0.0, 0.0, 0.0}, XSPHdv{0.0, 0.0, 0.0};
  Sym m2{0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#if SPH_FP64_SHARED_ACC
  // the two tensor sums (velocity gradient, M) accumulate in shared memory,
  // [component][thread]: 18 doubles per thread out of the register file
  __shared__ double sAcc[18][128];
  double* accDvDx = &sAcc[0][threadIdx.x];
  double* accM = &sAcc[9][threadIdx.x];
#pragma unroll
  for (int c = 0; c < 9; ++c) { accDvDx[128*c] = 0.0; accM[128*c] = 0.0; }
#else
  T9 DvDx{0, 0, 0, 0, 0, 0, 0, 0, 0}, M{0, 0, 0, 0, 0, 0, 0, 0, 0};
#endif
  // Cl *= 0.5*(fCli + fClj)*fshear (MonaghanGingoldViscosity::Piij), the Cl
  // and Cq multipliers 1; fshear = max of the two nodes' Balsara corrections,
  // else 1
  const double fsi = BALSARA ? MB.fshear[i] : 1.0;
  const int64_t k0 = offsets[i], k1 = offsets[i + 1];
  // node i's sums take the pair terms in row order
  auto accumulate = [&](const PairTerms& t, int64_t k) {
    wns += 1.0*fabs(t.gWI);
    {
      const double g2 = 1.0*mag2(t.gradWI);
      const Sym thpt = smul(selfdyad(t.rij), t.thptS);
      m2 = sadd(m2, smul(thpt, g2));
    }
    rhoSum += t.mj*t.WI;
    norm += I.mrho*t.WI;
    maxvp = dmax(maxvp, t.QI);
    effvp += t.mrhoj*t.QI*t.WI;
    viscW += t.mj*t.workQI;
    DvDt = vadd(DvDt, vmul(t.dd, t.own ? -t.mj : t.mj));
    DepsDt += t.mj*(t.PrhoI*dot(t.vij, t.gradWI) + t.workQI);
    if (COMPAT) {
      // the owner's pair acceleration, -m_other*deltaDvDt
      const V3 pa = vmul(t.dd, t.own ? -t.mj : -I.m);
      pacc[k] = pa.x;
      pacc[ecap + k] = pa.y;
      pacc[2*ecap + k] = pa.z;
    }
#if SPH_FP64_SHARED_ACC
    {
      // DvDx -= (vij gradW_i) m_j, element by element as tsubfrom(tmul(dyad))
      const double va[3] = {t.vij.x, t.vij.y, t.vij.z}, ga[3] = {t.gradWI.x, t.gradWI.y, t.gradWI.z};
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) accDvDx[128*(3*r + c)] = accDvDx[128*(3*r + c)] - (va[r]*ga[c])*t.mj;
    }
#else
    tsubfrom(DvDx, tmul(dyad(t.vij, t.gradWI), t.mj));
#endif
    if (XSPH) {
      const double w = 0.5*(I.mrho*t.WI + t.mrhoj*t.WJ);
      XSPHw += w;
      const V3 dvw = vmul(t.vij, w);
      XSPHdv = t.own ? vsub(XSPHdv, dvw) : vadd(XSPHdv, dvw);
    }
#if SPH_FP64_SHARED_ACC
    {
      const double ra[3] = {t.rij.x, t.rij.y, t.rij.z}, ga[3] = {t.gradWI.x, t.gradWI.y, t.gradWI.z};
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) accM[128*(3*r + c)] = accM[128*(3*r + c)] - (ra[r]*ga[c])*t.mj;
    }
#else
    tsubfrom(M, tmul(dyad(t.rij, t.gradWI), t.mj));
#endif
  };
  for (int64_t k = k0; k < k1; ++k) {
    const int32_t j = __ldg(nbr + k);
    const double fs = BALSARA ? dmax(fsi, MB.fshear[j < n ? (int64_t)j : (int64_t)MB.groot[j - n]]) : 1.0;
    accumulate(pairTerms<TENSILE>(I, isoI, loadRec(rec, j), j > (int32_t)i, P, P.Cl*(0.5*(1.0 + 1.0)*fs),
                                  P.Cq*(0.5*(1.0 + 1.0)*fs)), k);
  }

  // ---- per-node finish (src/SPH/SPHHydroBase.cc:834-902)
  const double mi = I.m, rhoi = I.rho, Hdeti = I.Hdet;
  const int numNeighbors = (int)(k1 - k0);
  rhoSum += mi*P.W0*Hdeti;
  norm += mi/rhoi*P.W0*Hdeti;
#if SPH_FP64_SHARED_ACC
  T9 Mi, DvDxi;
  {
    double* mi9 = &Mi.xx;
    double* dv9 = &DvDxi.xx;
#pragma unroll
    for (int c = 0; c < 9; ++c) { mi9[c] = accM[128*c]; dv9[c] = accDvDx[128*c]; }
  }
#else
  T9 Mi = M, DvDxi = DvDx;
#endif
  if (P.correctVelGrad && fabs(tdet(Mi)) > 1.0e-10 && numNeighbors > 8) {
    Mi = tinverse(Mi);
    DvDxi = tdot(DvDxi, Mi);
  } else {
    DvDxi = tdiv(DvDxi, rhoi);
  }
  const double DrhoDt = -rhoi*ttrace(DvDxi);
  wns = dmax(0.0, wns/Hdeti);
  wns = sgn(wns)*pow(fabs(wns), 0.3333333333333333);          // Dim<3>::rootnu
  m2 = sdiv(m2, Hdeti*Hdeti);
  V3 DxDt = I.v;
  if (XSPH) {
    XSPHw += Hdeti*mi/rhoi*P.W0;
    DxDt = vadd(I.v, vdiv(XSPHdv, dmax(1.0e-30, XSPHw)));
  }
  const Sym DHDt = smul(sdiv(sneg(I.H), 3.0), ttrace(DvDxi));
  // SPHSmoothingScale::idealSmoothingScale (src/NodeList/SPHSmoothingScale.cc:118-199)
  double nPerhCur;
  if (fuzzyEqual(wns, 0.0)) {
    nPerhCur = 0.5*P.nPerh;
  } else {
    nPerhCur = equivalentNodesPerSmoothingScale(P, wns);
  }
  const double s = dmin(4.0, dmax(0.25, P.nPerh/(nPerhCur + 1.0e-30)));
  const double a = s < 1.0 ? 0.4*(1.0 + s*s) : 0.4*(1.0 + 1.0/(s*s*s));
  const double hi0 = 1.0/I.H.xx;
  const double hi1 = dmin(P.hmax, dmax(P.hmin, hi0*(1.0 - a + a*s)));
  const double hinv = 1.0/hi1;

  // ---- stores (SoA, coalesced across the warp)
  double* d = D + i;
  d[(D_DXDT + 0)*n] = DxDt.x; d[(D_DXDT + 1)*n] = DxDt.y; d[(D_DXDT + 2)*n] = DxDt.z;
  d[(D_DVDT + 0)*n] = DvDt.x; d[(D_DVDT + 1)*n] = DvDt.y; d[(D_DVDT + 2)*n] = DvDt.z;
  d[D_DRHODT*n] = DrhoDt;
  d[D_DEPSDT*n] = DepsDt;
  d[(D_DHDT + 0)*n] = DHDt.xx; d[(D_DHDT + 1)*n] = DHDt.xy; d[(D_DHDT + 2)*n] = DHDt.xz;
  d[(D_DHDT + 3)*n] = DHDt.yy; d[(D_DHDT + 4)*n] = DHDt.yz; d[(D_DHDT + 5)*n] = DHDt.zz;
  d[(D_HIDEAL + 0)*n] = 1.0*hinv; d[(D_HIDEAL + 1)*n] = 0.0*hinv; d[(D_HIDEAL + 2)*n] = 0.0*hinv;
  d[(D_HIDEAL + 3)*n] = 1.0*hinv; d[(D_HIDEAL + 4)*n] = 0.0*hinv; d[(D_HIDEAL + 5)*n] = 1.0*hinv;
  const double* dv = &DvDxi.xx;
  const double* mm = &Mi.xx;
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    d[(D_DVDX + c)*n] = dv[c];
    d[(D_M + c)*n] = mm[c];
  }
  d[D_RHOSUM*n] = rhoSum;
  d[D_NORM*n] = norm;
  d[D_WNS*n] = wns;
  d[(D_M2 + 0)*n] = m2.xx; d[(D_M2 + 1)*n] = m2.xy; d[(D_M2 + 2)*n] = m2.xz;
  d[(D_M2 + 3)*n] = m2.yy; d[(D_M2 + 4)*n] = m2.yz; d[(D_M2 + 5)*n] = m2.zz;
  d[D_XSPHW*n] = XSPHw;
  d[(D_XSPHDV + 0)*n] = XSPHdv.x; d[(D_XSPHDV + 1)*n] = XSPHdv.y; d[(D_XSPHDV + 2)*n] = XSPHdv.z;
  d[D_MAXVP*n] = maxvp;
  d[D_EFFVP*n] = effvp;
  d[D_VISCW*n] = viscW;
}

// ---------------------------------------------------------------- grad-h
__global__ void __launch_bounds__(128) gradh_kernel(const Member* mem, BlockMap bm) {
  const MemberBlock mb = memberBlock(bm);
  const Member& MB = mem[mb.m];
  const int64_t n = MB.n;
  const int64_t i = mb.block*blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Params& P = MB.prm;
  const double* rec = MB.rec;
  const int32_t* nbr = MB.nbr;
  double* S = MB.S;
  const int64_t k0 = MB.offsets[i], k1 = MB.offsets[i + 1];
  if (k1 == k0) { S[S_OMEGA*n + i] = 1.0; return; }
  const Rec I = loadRec(rec, i);
  const double W0 = tableKernel(P.W, 0.0, I.Hdet);
  double omega = 0.0, gradsum = 0.0;
  bool selfDone = false;
  for (int64_t k = k0; k < k1; ++k) {
    const int32_t j = __ldg(nbr + k);
    if (!selfDone && j > (int32_t)i) { omega += W0; selfDone = true; }
    const V3 rj{ldg(rec + (int64_t)j*RECW + R_X), ldg(rec + (int64_t)j*RECW + R_Y), ldg(rec + (int64_t)j*RECW + R_Z)};
    const V3 rij = vsub(I.r, rj);
    const double eta = mag(sdot(I.H, rij));
    double W, gW;
    tableKernelAndGrad(P.W, eta, I.Hdet, W, gW);
    omega += W;
    gradsum += eta*gW;
  }
  if (!selfDone) omega += W0;
  S[S_OMEGA*n + i] = -gradsum/(3*omega);
}

// ---------------------------------------------------------------- sum density
// PeriodicBoundary::enforceBoundary (src/Boundary/PeriodicBoundary.cc:145-203)
// for one internal node's position.
__device__ __forceinline__ V3 enforcedPosition(const BoxBCs& bcs, V3 r) {
  for (int pb = 0; pb < 6; pb += 2) {
    if (!bcs.periodic[pb >> 1]) continue;
    for (int sub = 0; sub < 2; ++sub) {
      const PlanarBC& bc = bcs.bc[pb + sub];
      if (planeCompare(bc.enter, r) == 1) r = mapPositionThroughPlanes(r, bc.enter, bc.exit);
    }
    const PlaneD& plane1 = bcs.bc[pb].enter;
    const PlaneD& plane2 = bcs.bc[pb].exit;
    if (planeCompare(plane1, r) == 1 || planeCompare(plane2, r) == 1) {
      const double L = minimumDistance(plane1, plane2.point);
      const V3 p0 = vadd(r, vmul(plane1.normal, dot(vsub(plane1.point, r), plane1.normal)));
      const double f = dmax(-1.0, dmin(1.0, fmod(signedDistance(plane1, r)/L, 1.0)));
      r = vadd(p0, vmul(plane1.normal, f*L));
    }
  }
  return r;
}

__device__ __forceinline__ void enforceNode(const Member& MB, int64_t i) {
  double* S = MB.S;
  const int64_t n = MB.n;
  const V3 r = enforcedPosition(MB.prm.bcs, V3{S[S_X*n + i], S[S_Y*n + i], S[S_Z*n + i]});
  S[S_X*n + i] = r.x; S[S_Y*n + i] = r.y; S[S_Z*n + i] = r.z;
}

// enforce: also wrap the node's position through the periodic planes (the
// step's enforceBoundaries, which follows the summed density; the pair
// terms read positions from the records, never from the state)
__global__ void __launch_bounds__(128) sum_density_kernel(const Member* mem, BlockMap bm, int enforce) {
  const MemberBlock mb = memberBlock(bm);
  const Member& MB = mem[mb.m];
  const int64_t n = MB.n;
  const int64_t i = mb.block*blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Params& P = MB.prm;
  const double* rec = MB.rec;
  const int32_t* nbr = MB.nbr;
  const V3 ri{ldg(rec + i*RECW + R_X), ldg(rec + i*RECW + R_Y), ldg(rec + i*RECW + R_Z)};
  const double mi = ldg(rec + i*RECW + R_M), Hdeti = ldg(rec + i*RECW + R_HDET);
  const double W0 = tableKernel(P.W, 0.0, Hdeti);
  double rho = 0.0;
  bool selfDone = false;
  const int64_t k0 = MB.offsets[i], k1 = MB.offsets[i + 1];
  for (int64_t k = k0; k < k1; ++k) {
    const int32_t j = __ldg(nbr + k);
    if (!selfDone && j > (int32_t)i) { rho += mi*W0; selfDone = true; }
    const Rec J = loadRec(rec, j);
    const V3 rij = vsub(ri, J.r);
    const double eta = mag(isoSym(J.H) ? vmul(rij, J.H.xx) : sdot(J.H, rij));
    rho += J.m*tableKernel(P.W, eta, J.Hdet);
  }
  if (!selfDone) rho += mi*W0;
  MB.S[S_RHO*n + i] = rho;
  if (enforce) enforceNode(MB, i);
}

// ---------------------------------------------------------------- summed density, mixed form
struct KahanSum {
  float s, c;
  __device__ __forceinline__ void add(float x) {
    const float y = x - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
  }
  __device__ __forceinline__ double value() const { return (double)s - (double)c; }
};

// FP32 TableKernel value (the FP32 copy of the coefficient table).
__device__ __forceinline__ float tableW32(const float* coef, int n, float invStep, float extent, float eta,
                                          float Hdet) {
  if (!(eta < extent)) return 0.0f;
  const float q = eta*invStep;
  int lb = (int)q;
  lb = lb < n - 1 ? lb : n - 1;
  const int i0 = lb < n - 3 ? lb : n - 3;
  const float x = q - (float)i0;
  const float2* c = reinterpret_cast<const float2*>(coef + 6*(i0 + 1));
  const float2 c01 = __ldg(c), c23 = __ldg(c + 1);
  return Hdet*(c01.x + x*(c01.y + x*c23.x));
}

// computeSPHSumMassDensity (src/SPH/computeSPHSumMassDensity.cc:27-111),
// RigorousSumDensity, mixed form: rho_i = m_i W(0) + sum_j m_j W(|H_j r_ij|)
// with the pair terms in FP32 (r_ij formed in FP64, rounded once) and a
// Kahan-compensated FP32 sum, from the mixed records of the end-of-step
// state.  enforce as for sum_density_kernel.
__global__ void __launch_bounds__(128) sum_density_mixed_kernel(const Member* mem, BlockMap bm, int enforce) {
  const MemberBlock mb = memberBlock(bm);
  const Member& MB = mem[mb.m];
  const int64_t n = MB.n;
  const int64_t i = mb.block*blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Params& P = MB.prm;
  const float* coefF = MB.coefF;
  const double* mrec = MB.mrec;
  const int32_t* nbr = MB.nbr;
  const float invStep = (float)(1.0/P.W.stepSize), extent = (float)P.W.extent;
  const double2* qi = reinterpret_cast<const double2*>(mrec + i*MRECW);
  const double2 a0 = __ldg(qi), a1 = __ldg(qi + 1);
  const float4 bi = __ldg(reinterpret_cast<const float4*>(qi + 3));
  const float W0 = tableW32(coefF, P.W.n, invStep, extent, 0.0f, bi.w);
  KahanSum rho{0.0f, 0.0f};
  bool selfDone = false;
  const int64_t k0 = MB.offsets[i], k1 = MB.offsets[i + 1];
  for (int64_t k = k0; k < k1; ++k) {
    const int32_t j = __ldg(nbr + k);
    if (!selfDone && j > (int32_t)i) { rho.add(bi.x*W0); selfDone = true; }
    const double2* q = reinterpret_cast<const double2*>(mrec + (int64_t)j*MRECW);
    const double2 c0 = __ldg(q), c1 = __ldg(q + 1);
    const float4* f = reinterpret_cast<const float4*>(q + 3);
    const float4 f0 = __ldg(f), f1 = __ldg(f + 1);
    const float2 f2 = __ldg(reinterpret_cast<const float2*>(f + 2));
    const float rx = (float)(a0.x - c0.x), ry = (float)(a0.y - c0.y), rz = (float)(a1.x - c1.x);
    const float ex = f1.x*rx + f1.y*ry + f1.z*rz;
    const float ey = f1.y*rx + f1.w*ry + f2.x*rz;
    const float ez = f1.z*rx + f2.x*ry + f2.y*rz;
    const float eta = sqrtf(ex*ex + ey*ey + ez*ez);
    rho.add(f0.x*tableW32(coefF, P.W.n, invStep, extent, eta, f0.w));
  }
  if (!selfDone) rho.add(bi.x*W0);
  MB.S[S_RHO*n + i] = rho.value();
  if (enforce) enforceNode(MB, i);
}

// ---------------------------------------------------------------- compatible energy
// SpecificThermalEnergyPolicy::update (src/Hydro/SpecificThermalEnergyPolicy.cc:66-189,
// compatible energy) for internal node i: the energy increment rate from the
// owner-oriented pair accelerations, with the half-step velocities
// v + a dt/2 of the start-of-step state S0 and the weights |DepsDt| + eps.
// Evaluated in the full RK2 update, where the reference has restored state0.
__device__ __forceinline__ double compatibleDepsDt(const Member& MB, int64_t i, double hdt) {
  const int64_t n = MB.n;
  const double* D = MB.D;
  const double* S = MB.S;
  const double* S0 = MB.S0;
  const int32_t* nbr = MB.nbr;
  const int32_t* groot = MB.groot;
  const double* pacc = MB.pacc;
  const float* paccF = reinterpret_cast<const float*>(MB.pacc);
  const bool mixed = MB.prm.precision == SPHGPU_PRECISION_MIXED;
  const int64_t ecap = MB.ecap;
  const double weighti = fabs(D[D_DEPSDT*n + i]) + kDblEps;
  const double mi = S[S_M*n + i];                // mass is constant within the step
  const V3 vi{S0[S_VX*n + i], S0[S_VY*n + i], S0[S_VZ*n + i]};
  const V3 ai{D[(D_DVDT + 0)*n + i], D[(D_DVDT + 1)*n + i], D[(D_DVDT + 2)*n + i]};
  const V3 vi12 = vadd(vi, vmul(ai, hdt));
  double DepsDti = 0.0;
  const int64_t k0 = MB.offsets[i], k1 = MB.offsets[i + 1];
  for (int64_t k = k0; k < k1; ++k) {
    const int32_t j = __ldg(nbr + k);
    const int64_t r = j < n ? (int64_t)j : (int64_t)__ldg(groot + (j - n));
    const double weightj = fabs(ldg(D + D_DEPSDT*n + r)) + kDblEps;
    const double mj = ldg(S + S_M*n + r);
    const V3 vj{ldg(S0 + S_VX*n + r), ldg(S0 + S_VY*n + r), ldg(S0 + S_VZ*n + r)};
    const V3 aj{ldg(D + (D_DVDT + 0)*n + r), ldg(D + (D_DVDT + 1)*n + r), ldg(D + (D_DVDT + 2)*n + r)};
    const V3 vj12 = vadd(vj, vmul(aj, hdt));
    // owner's pair acceleration (FP32 in the mixed form)
    const V3 pa = mixed ? V3{(double)__ldg(paccF + k), (double)__ldg(paccF + ecap + k), (double)__ldg(paccF + 2*ecap + k)}
                        : V3{ldg(pacc + k), ldg(pacc + ecap + k), ldg(pacc + 2*ecap + k)};
    if (j > (int32_t)i) {
      const double duij = dot(vsub(vj12, vi12), pa);
      const double wi = weighti/(weighti + weightj);
      DepsDti += wi*duij;
    } else {
      const double duji = dot(vsub(vi12, vj12), pa);
      const double wj = weightj/(weightj + weighti);
      DepsDti += (1.0 - wj)*duji*mj/mi;
    }
  }
  return DepsDti;
}

// ---------------------------------------------------------------- policies
// The bounded H policies: min(1/hmin, max(1/hmax, H)) with the eigenvalue
// limiters (boundedSym).  When the Gershgorin discs of H lie inside
// (1/hmax, 1/hmin) with a relative margin far above the eigen solve's
// rounding, every eigenvalue does and the reference returns H unchanged;
// only the other tensors take the eigen solve.
__device__ __forceinline__ Sym boundH(const Sym& H, double hmin, double hmax) {
  const double rx = dabs(H.xy) + dabs(H.xz), ry = dabs(H.xy) + dabs(H.yz), rz = dabs(H.xz) + dabs(H.yz);
  const double glo = dmin(H.xx - rx, dmin(H.yy - ry, H.zz - rz));
  const double ghi = dmax(H.xx + rx, dmax(H.yy + ry, H.zz + rz));
  if (glo > (1.0/hmax)*(1.0 + 1.0e-12) && ghi < (1.0/hmin)*(1.0 - 1.0e-12)) return H;
  return boundedSym(H, 1.0/hmax, 1.0/hmin);
}

// State::update of every policy, f = f_src + scale*dt*df, into S.
// UPDATE_IN_PLACE: the source is S.  UPDATE_SAVE_START: the source is S,
// saved to S0 first (state0 = state.copyState()).  UPDATE_FROM_START: the
// source is S0 (state.assign(state0) fused into the update); with
// compatible energy the specific thermal energy comes from
// compatibleDepsDt (its pair loop reads S0 and the derivatives only, which
// no thread of this launch writes).  S0 holds only what the rest of the step reads from
// it: position, velocity, density, energy, H, plus omega with grad-h (the
// mid-point initialize changes it) and the CRKSPH volume.  Mass is constant
// and pressure and sound speed are recomputed, so S0 skips them.
// packMode 1 / 2 also writes the node's pair record for the mid-point
// evaluation / the end-of-step summed density (SPH members, see
// packedByUpdate).
// recordMid (the RK2 step, with packMode 1 in the mid-point update): for the
// members whose mid-point records the update writes (SPH without grad-h) the
// mid-point state lives in those records only.  The mid-point update leaves
// S at the start of the step and writes to S0 only the start velocity (the
// compatible energy's pair loop reads it while the full update overwrites
// S) and the mid-point H and mass density (the mixed pair kernel's FP64
// finish reads them, sph_eval_mixed_kernel's midInS0); the full update then
// reads its source state from S.
enum UpdateMode { UPDATE_IN_PLACE = 0, UPDATE_SAVE_START = 1, UPDATE_FROM_START = 2 };

// COMPAT: the launch applies the compatible energy of its compatible members
// (only from the start-of-step state: mode UPDATE_FROM_START, the full update
// of the RK2 step); a separate instance keeps the pair loop's registers out of
// the other updates.
#ifndef SPH_UPDATE_MIN_BLOCKS
#define SPH_UPDATE_MIN_BLOCKS 6
#endif
template<bool COMPAT>
__global__ void __launch_bounds__(128, SPH_UPDATE_MIN_BLOCKS) update_kernel(const Member* mem, BlockMap bm, double scale,
                                                     int timeAdvanceOnly, int mode, int packMode, int recordMid) {
  const MemberBlock mb = memberBlock(bm);
  const Member& MB = mem[mb.m];
  const int64_t n = MB.n;
  const int64_t i = mb.block*blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Params& P = MB.prm;
  const double mult = scale*MB.scal[SC_DT];
  // the compatible energy's pair loop first, before the node's fields are live
  const bool compatible = COMPAT && P.compatible;
  const double compatDeps = compatible ? compatibleDepsDt(MB, i, 0.5*mult) : 0.0;
  double* S = MB.S;
  double* S0 = MB.S0;
  const double* D = MB.D;
  const bool crk = P.hydro == SPHGPU_HYDRO_CRKSPH;
  // (grad-h changes omega and the Balsara correction reads the mid-point H
  // and sound speed after this update: those members keep the state in S)
  const bool recMid = recordMid && !crk && !P.gradh && !P.balsara;
  const bool midInRecords = recMid && mode == UPDATE_SAVE_START;   // S keeps the start state
  const double* Src = mode == UPDATE_FROM_START && !recMid ? S0 : S;
  // the source state of the updated fields
  V3 x{Src[S_X*n + i], Src[S_Y*n + i], Src[S_Z*n + i]};
  V3 v{Src[S_VX*n + i], Src[S_VY*n + i], Src[S_VZ*n + i]};
  const double rho0 = Src[S_RHO*n + i];
  const double eps0 = Src[S_EPS*n + i];
  const Sym H{Src[(S_H + 0)*n + i], Src[(S_H + 1)*n + i], Src[(S_H + 2)*n + i],
              Src[(S_H + 3)*n + i], Src[(S_H + 4)*n + i], Src[(S_H + 5)*n + i]};
  const double vol0 = crk ? Src[S_VOL*n + i] : 0.0;
  if (midInRecords) {
    S0[S_VX*n + i] = v.x; S0[S_VY*n + i] = v.y; S0[S_VZ*n + i] = v.z;
  } else if (mode == UPDATE_SAVE_START) {
    S0[S_X*n + i] = x.x; S0[S_Y*n + i] = x.y; S0[S_Z*n + i] = x.z;
    S0[S_VX*n + i] = v.x; S0[S_VY*n + i] = v.y; S0[S_VZ*n + i] = v.z;
    S0[S_RHO*n + i] = rho0;
    S0[S_EPS*n + i] = eps0;
    S0[(S_H + 0)*n + i] = H.xx; S0[(S_H + 1)*n + i] = H.xy; S0[(S_H + 2)*n + i] = H.xz;
    S0[(S_H + 3)*n + i] = H.yy; S0[(S_H + 4)*n + i] = H.yz; S0[(S_H + 5)*n + i] = H.zz;
    if (P.gradh) S0[S_OMEGA*n + i] = S[S_OMEGA*n + i];
    if (crk) S0[S_VOL*n + i] = vol0;
  } else if (mode == UPDATE_FROM_START && P.gradh) {
    S[S_OMEGA*n + i] = S0[S_OMEGA*n + i];
  }
  // H: IncrementBoundedState (half step / IntegrateH) or ReplaceBoundedState (IdealH)
  Sym Hn;
  if (timeAdvanceOnly || P.HUpdate == SPHGPU_H_INTEGRATE) {
    const Sym dH{D[(D_DHDT + 0)*n + i], D[(D_DHDT + 1)*n + i], D[(D_DHDT + 2)*n + i],
                 D[(D_DHDT + 3)*n + i], D[(D_DHDT + 4)*n + i], D[(D_DHDT + 5)*n + i]};
    Hn = sadd(H, smul(dH, mult));
  } else {
    Hn = Sym{D[(D_HIDEAL + 0)*n + i], D[(D_HIDEAL + 1)*n + i], D[(D_HIDEAL + 2)*n + i],
             D[(D_HIDEAL + 3)*n + i], D[(D_HIDEAL + 4)*n + i], D[(D_HIDEAL + 5)*n + i]};
  }
  Hn = boundH(Hn, P.hmin, P.hmax);
  double* SH = midInRecords ? S0 : S;                // where the new H and mass density go
  SH[(S_H + 0)*n + i] = Hn.xx; SH[(S_H + 1)*n + i] = Hn.xy; SH[(S_H + 2)*n + i] = Hn.xz;
  SH[(S_H + 3)*n + i] = Hn.yy; SH[(S_H + 4)*n + i] = Hn.yz; SH[(S_H + 5)*n + i] = Hn.zz;
  // mass density: IncrementBoundedState
  const double drho = D[D_DRHODT*n + i];
  const double rho = dmin(P.rhoMax, dmax(P.rhoMin, rho0 + mult*(drho)));
  SH[S_RHO*n + i] = rho;
  // position: IncrementFieldList
  x = V3{x.x + D[(D_DXDT + 0)*n + i]*mult, x.y + D[(D_DXDT + 1)*n + i]*mult, x.z + D[(D_DXDT + 2)*n + i]*mult};
  if (!midInRecords) { S[S_X*n + i] = x.x; S[S_Y*n + i] = x.y; S[S_Z*n + i] = x.z; }
  const double m = S[S_M*n + i];                     // constant within the step
  // CRKSPH node volume: ContinuityVolumePolicy (after mass density and H)
  if (crk) {
    const double volMin = 0.5*m*safeInvVar(rho);
    const double volMax = 4.0*3.14159265358979323846/(3.0*sdet(Hn));
    const double dVdt = -m*safeInvVar(rho*rho)*drho;
    S[S_VOL*n + i] = dmax(volMin, dmin(volMax, vol0 + mult*dVdt));
  }
  // specific thermal energy: IncrementFieldList, or the compatible policy
  // (from the start-of-step state: only in the full update)
  const double eps = compatible ? eps0 + compatDeps*mult : eps0 + mult*(D[D_DEPSDT*n + i]);
  // pressure, sound speed (GammaLawGas, no active pressure limits)
  const double g1 = P.gamma - 1.0;
  const double Pn = g1*rho*eps;
  const double csn = sqrt(dmax(0.0, P.gamma*g1*eps));
  // velocity: IncrementFieldList (after the energy it depends on)
  v = V3{v.x + D[(D_DVDT + 0)*n + i]*mult, v.y + D[(D_DVDT + 1)*n + i]*mult, v.z + D[(D_DVDT + 2)*n + i]*mult};
  if (mode == UPDATE_FROM_START) {
    // the start-of-step energy the reference's state0 leaves in its
    // specificThermalEnergy0 (compatible energy; members that read their
    // source from S0 have it there already)
    if (P.compatible && Src == S) S0[S_EPS*n + i] = eps0;
    // CRKSPH's EntropyPolicy (src/Hydro/EntropyPolicy.cc:52-82):
    // GammaLawGas::setEntropy of the updated density and energy
    if (crk) S0[S0_ENTROPY*n + i] = Pn*safeInvVar(pow(rho, P.gamma));
  }
  if (!midInRecords) {
    S[S_EPS*n + i] = eps;
    S[S_P*n + i] = Pn;
    S[S_CS*n + i] = csn;
    S[S_VX*n + i] = v.x; S[S_VY*n + i] = v.y; S[S_VZ*n + i] = v.z;
  }
  // the internal node's record for the next pair loop, from the new state
  const bool pack = packMode != 0 && !crk &&
                    (packMode == 1 ? !P.gradh : P.densityUpdate == SPHGPU_DENSITY_RIGOROUS_SUM);
  if (pack) {
    const double omega = S[S_OMEGA*n + i];
    if (P.precision == SPHGPU_PRECISION_MIXED) writeMixedRecord(MB.mrec, i, x, v, m, rho, csn, Pn, omega, Hn);
    else writeRecord(MB.rec, i, x, v, m, rho, csn, Pn, omega, Hn);
  }
}

__global__ void __launch_bounds__(256) eos_kernel(const Member* mem, BlockMap bm) {
  const MemberBlock mb = memberBlock(bm);
  const Member& MB = mem[mb.m];
  const int64_t n = MB.n;
  const int64_t i = mb.block*blockDim.x + threadIdx.x;
  if (i >= n) return;
  double* S = MB.S;
  const double gamma = MB.prm.gamma;
  const double g1 = gamma - 1.0;
  const double rho = S[S_RHO*n + i], eps = S[S_EPS*n + i];
  S[S_P*n + i] = g1*rho*eps;
  S[S_CS*n + i] = sqrt(dmax(0.0, gamma*g1*eps));
}

// PeriodicBoundary::enforceBoundary over every internal node of the members
__global__ void __launch_bounds__(256) enforce_boundaries_kernel(const Member* mem, BlockMap bm) {
  const MemberBlock mb = memberBlock(bm);
  const Member& MB = mem[mb.m];
  const int64_t i = mb.block*blockDim.x + threadIdx.x;
  if (i >= MB.n) return;
  enforceNode(MB, i);
}

// ---------------------------------------------------------------- iterateIdealH
// One iteration of iterateIdealH (src/Utilities/iterateIdealH.cc:26-349, the
// drivers' arguments: nPerhForIteration 0, no spherical start, no fixed
// determinant) with SPHSmoothingScale::idealSmoothingScale
// (src/NodeList/SPHSmoothingScale.cc:102-225), one thread per internal node
// over its ascending CSR row.  Nodes whose last change was within the
// tolerance keep their H.  H is replaced in place: the moment of node i
// reads only its own H and the positions.  deltaH[i] receives
// max |eig((H1^1/2 Hi^-1 H1^1/2).Symmetric()) - 1|; H1 = c I, whose square
// root the reference takes from a diagonal eigen decomposition (eigenvalue
// (c*(1/c))*c, identity eigenvectors).  The largest change goes to
// SC_DELTAH.
__global__ void __launch_bounds__(128) ideal_h_iter_kernel(const Member* mem, BlockMap bm, double tolerance,
                                                            double* deltaH) {
  const MemberBlock mb = memberBlock(bm);
  const Member& MB = mem[mb.m];
  const int64_t n = MB.n;
  const int64_t i = mb.block*blockDim.x + threadIdx.x;
  double dHi = 0.0;
  if (i < n && deltaH[i] > tolerance) {
    const Params& P = MB.prm;
    double* S = MB.S;
    const V3 ri{S[S_X*n + i], S[S_Y*n + i], S[S_Z*n + i]};
    const Sym Hi{S[(S_H + 0)*n + i], S[(S_H + 1)*n + i], S[(S_H + 2)*n + i],
                 S[(S_H + 3)*n + i], S[(S_H + 4)*n + i], S[(S_H + 5)*n + i]};
    double zerothMoment = 0.0;
    const int64_t k0 = MB.offsets[i], k1 = MB.offsets[i + 1];
    for (int64_t k = k0; k < k1; ++k) {
      const int32_t j = __ldg(MB.nbr + k);
      V3 rj;
      if (j < n) rj = V3{ldg(S + S_X*n + j), ldg(S + S_Y*n + j), ldg(S + S_Z*n + j)};
      else rj = V3{ldg(MB.gpos + (j - n)), ldg(MB.gpos + MB.gcap + (j - n)), ldg(MB.gpos + 2*MB.gcap + (j - n))};
      const V3 xij = vsub(ri, rj);
      const double etai = mag(sdot(Hi, xij));
      double W, gW;
      tableKernelAndGrad(P.W, etai, 1.0, W, gW);
      zerothMoment += dabs(gW);
    }
    zerothMoment = sgn(zerothMoment)*pow(dabs(zerothMoment), 0.3333333333333333);   // Dim<3>::rootnu
    double nPerhCur;
    if (fuzzyEqual(zerothMoment, 0.0)) nPerhCur = 0.5*P.nPerh;
    else nPerhCur = equivalentNodesPerSmoothingScale(P, zerothMoment);
    const double s = dmin(4.0, dmax(0.25, P.nPerh/(nPerhCur + 1.0e-30)));
    const double a = s < 1.0 ? 0.4*(1.0 + s*s) : 0.4*(1.0 + 1.0/(s*s*s));
    const double hi0 = 1.0/Hi.xx;
    const double hi1 = dmin(P.hmax, dmax(P.hmin, hi0*(1.0 - a + a*s)));
    const double inv = 1.0/hi1;
    const Sym H1{1.0*inv, 0.0*inv, 0.0*inv, 1.0*inv, 0.0*inv, 1.0*inv};
    const double fscale = dmax(10.0*kDblEps, smaxAbs(H1));
    const double r = sqrt((inv*(1.0/fscale))*fscale);
    const Sym Hinv = sinverse(Hi);
    const Sym T{r*(r*Hinv.xx), r*(r*Hinv.xy), r*(r*Hinv.xz), r*(r*Hinv.yy), r*(r*Hinv.yz), r*(r*Hinv.zz)};
    const V3 phi = eigenValues(T);
    dHi = dmax(dabs(vmin(phi) - 1.0), dabs(vmax(phi) - 1.0));
    deltaH[i] = dHi;
    S[(S_H + 0)*n + i] = H1.xx; S[(S_H + 1)*n + i] = H1.xy; S[(S_H + 2)*n + i] = H1.xz;
    S[(S_H + 3)*n + i] = H1.yy; S[(S_H + 4)*n + i] = H1.yz; S[(S_H + 5)*n + i] = H1.zz;
  }
  for (int o = 16; o > 0; o >>= 1) dHi = dmax(dHi, __shfl_xor_sync(0xffffffffu, dHi, o));
  if ((threadIdx.x & 31) == 0 && dHi > 0.0)
    atomicMax(reinterpret_cast<unsigned long long*>(MB.scal + SC_DELTAH), (unsigned long long)__double_as_longlong(dHi));
}

// ---------------------------------------------------------------- dt
// cachedEig: max eig(H) of each node is the one the neighbor build stored
// (hmaxi[n + i]), valid when H has not changed since that build (the step's
// selectDt, which follows the build); otherwise it is solved here.
__global__ void __launch_bounds__(128) hydro_dt_kernel(const Member* mem, BlockMap bm, int slot, int cachedEig) {
  const MemberBlock mb = memberBlock(bm);
  const Member& MB = mem[mb.m];
  const int64_t n = MB.n;
  const int64_t i = mb.block*blockDim.x + threadIdx.x;
  const Params& P = MB.prm;
  const double* S = MB.S;
  const double* D = MB.D;
  double minDt = kFltMax;
  if (i < n) {
    double lmax;
    if (cachedEig) {
      lmax = MB.hmaxi[n + i];
    } else {
      const Sym H{S[(S_H + 0)*n + i], S[(S_H + 1)*n + i], S[(S_H + 2)*n + i],
                  S[(S_H + 3)*n + i], S[(S_H + 4)*n + i], S[(S_H + 5)*n + i]};
      lmax = vmax(eigenValues(H));
    }
    const double nodeScale = 1.0/lmax/P.nPerh;
    const double cs = S[S_CS*n + i], rho = S[S_RHO*n + i];
    const double csDt = nodeScale/(cs + kFltMin);
    if (csDt < minDt) minDt = csDt;
    const double csq = sqrt(D[D_MAXVP*n + i]/rho);
    const double csqDt = nodeScale/(csq + kFltMin);
    if (csqDt < minDt) minDt = csqDt;
    const double divv = D[(D_DVDX + 0)*n + i] + D[(D_DVDX + 4)*n + i] + D[(D_DVDX + 8)*n + i];
    const double divvDt = 1.0/(fabs(divv) + kFltMin);
    if (divvDt < minDt) minDt = divvDt;
    const V3 vi{S[S_VX*n + i], S[S_VY*n + i], S[S_VZ*n + i]};
    // min over the neighbors of nodeScale*safeInvVar(|vi - vj|): sqrt and the
    // division are correctly rounded and monotone, so it is the term of the
    // largest |vi - vj|^2, one sqrt and one division per node (bit-identical)
    double v2max = -1.0;
    for (int64_t k = MB.offsets[i]; k < MB.offsets[i + 1]; ++k) {
      const int32_t j = __ldg(MB.nbr + k);
      const int64_t r = j < n ? (int64_t)j : (int64_t)__ldg(MB.groot + (j - n));
      const V3 vj{ldg(S + S_VX*n + r), ldg(S + S_VY*n + r), ldg(S + S_VZ*n + r)};
      const V3 d = vsub(vi, vj);
      const double v2 = d.x*d.x + d.y*d.y + d.z*d.z;
      if (v2 > v2max) v2max = v2;
    }
    if (v2max >= 0.0) {
      const double dtVelDiff = nodeScale*safeInvVar(sqrt(v2max), 1e-30);
      if (dtVelDiff < minDt) minDt = dtVelDiff;
    }
    const V3 a{D[(D_DVDT + 0)*n + i], D[(D_DVDT + 1)*n + i], D[(D_DVDT + 2)*n + i]};
    const double dtAcc = sqrt(nodeScale/(mag(a) + kFltMin));
    if (dtAcc < minDt) minDt = dtAcc;
    if (P.useVelMagDt) {
      const double velDt = nodeScale/(mag(vi) + 1.0e-10);
      if (velDt < minDt) minDt = velDt;
    }
  }
  for (int o = 16; o > 0; o >>= 1) minDt = dmin(minDt, __shfl_xor_sync(0xffffffffu, minDt, o));
  if ((threadIdx.x & 31) == 0)
    atomicMin(reinterpret_cast<unsigned long long*>(MB.scal + slot), (unsigned long long)__double_as_longlong(minDt));
}

// Integrator::selectDt on the device: dt stays resident for the step kernels.
__global__ void select_dt_kernel(const Member* mem, int nmem) {
  const int m = blockIdx.x*blockDim.x + threadIdx.x;
  if (m >= nmem) return;
  const Params& P = mem[m].prm;
  double* sc = mem[m].scal;
  const double vote = P.cfl*sc[SC_MINDT];
  double dt = P.dtMax;
  if (vote > 0.0 && vote < dt) dt = vote;
  dt = dmin(dt, P.dtGrowth*sc[SC_LASTDT]);
  dt = dmin(P.dtMax, dmax(P.dtMin, dt));
  sc[SC_DT] = dt;
  sc[SC_VOTE] = vote;
}

// End of a completed step: last dt, and the step bookkeeping a graph replay
// reads back only at the end of a call (time += dt as the integrator does,
// steps and pair interactions counted).
__global__ void finish_step_kernel(const Member* mem, int nmem) {
  const int m = blockIdx.x*blockDim.x + threadIdx.x;
  if (m >= nmem) return;
  double* s = mem[m].scal;
  const double dt = s[SC_DT];
  s[SC_LASTDT] = dt;
  s[SC_TIME] = s[SC_TIME] + dt;
  int64_t* si = reinterpret_cast<int64_t*>(s);
  si[SC_STEPS] += 1;
  si[SC_PAIRSUM] += si[SC_PAIRS];
}

// ---------------------------------------------------------------- conservation
// Fixed partition per member (grid-stride over its blocks), fixed-order
// reduction: the sums are reproducible.  The total energy is also summed as
// a double-double (Knuth's two-sum: each addition's rounding error is kept in
// a second double), so that drifts far below the rounding of a plain FP64
// sum over millions of nodes can be read: out[6] + out[7] is the total to
// about 2^-100 relative, out[6] alone its rounded value.
__device__ __forceinline__ void twoSumAdd(double& hi, double& lo, double x) {
  const double s = hi + x;
  const double bb = s - hi;
  const double err = (hi - (s - bb)) + (x - bb);
  hi = s;
  lo += err;
}

__global__ void __launch_bounds__(256) conservation_partials_kernel(const Member* mem, BlockMap bm) {
  const MemberBlock mb = memberBlock(bm);
  const Member& MB = mem[mb.m];
  const int64_t n = MB.n;
  const double* S = MB.S;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int64_t i = mb.block*blockDim.x + threadIdx.x; i < n; i += (int64_t)mb.blocks*blockDim.x) {
    const double m = S[S_M*n + i];
    const V3 v{S[S_VX*n + i], S[S_VY*n + i], S[S_VZ*n + i]};
    const double ke = 0.5*m*mag2(v), te = m*S[S_EPS*n + i];
    acc[0] += m;
    acc[1] += m*v.x; acc[2] += m*v.y; acc[3] += m*v.z;
    acc[4] += ke;
    acc[5] += te;
    twoSumAdd(acc[6], acc[7], ke);
    twoSumAdd(acc[6], acc[7], te);
  }
  __shared__ double sh[8][256];
  for (int c = 0; c < 8; ++c) sh[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int s = blockDim.x/2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      for (int c = 0; c < 6; ++c) sh[c][threadIdx.x] += sh[c][threadIdx.x + s];
      double hi = sh[6][threadIdx.x], lo = sh[7][threadIdx.x] + sh[7][threadIdx.x + s];
      twoSumAdd(hi, lo, sh[6][threadIdx.x + s]);
      sh[6][threadIdx.x] = hi;
      sh[7][threadIdx.x] = lo;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) for (int c = 0; c < 8; ++c) MB.red[mb.block*8 + c] = sh[c][0];
}

__global__ void conservation_final_kernel(const Member* mem, int nmem, const int32_t* partialBlocks, int soloBlocks) {
  const int m = blockIdx.x*blockDim.x + threadIdx.x;
  if (m >= nmem) return;
  const Member& MB = mem[m];
  const int nb = partialBlocks ? partialBlocks[m + 1] - partialBlocks[m] : soloBlocks;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  double hi = 0.0, lo = 0.0;
  for (int b = 0; b < nb; ++b) {
    for (int c = 0; c < 6; ++c) acc[c] += MB.red[b*8 + c];
    lo += MB.red[b*8 + 7];
    twoSumAdd(hi, lo, MB.red[b*8 + 6]);
  }
  // renormalise: hi the rounded total, lo what it leaves out
  const double s = hi + lo;
  const double e = lo - (s - hi);
  double* out = MB.scal + SC_CONS;
  for (int c = 0; c < 6; ++c) out[c] = acc[c];
  out[6] = s;
  out[7] = e;
}

__global__ void __launch_bounds__(256) zero_derivs_kernel(const Member* mem, BlockMap bm) {
  const MemberBlock mb = memberBlock(bm);
  const Member& MB = mem[mb.m];
  const int64_t k = mb.block*blockDim.x + threadIdx.x;
  if (k < NDERIV*MB.n) MB.D[k] = 0.0;
}

}  // namespace

// ================================================================ launchers
namespace {

bool isSph(const Problem& p) { return p.prm.hydro == SPHGPU_HYDRO_SPH; }
bool isFp64Sph(const Problem& p) { return isSph(p) && p.cfg.precision == SPHGPU_PRECISION_FP64; }

int map_nodes(Batch& b, int threads, BlockMap* bm, unsigned* grid) {
  return batch_map_items(b, [](const Problem& p) { return p.n; }, threads, bm, grid);
}


}  // namespace

bool packedByUpdate(const Problem& p, int packMode) {
  if (p.prm.hydro != SPHGPU_HYDRO_SPH) return false;
  if (packMode == PACK_FOR_EVAL) return !p.prm.gradh;               // grad-h changes omega after the update
  if (packMode == PACK_FOR_FINALIZE) return p.prm.densityUpdate == SPHGPU_DENSITY_RIGOROUS_SUM;
  return false;
}

namespace {

// Records of every node (full) or of the ghosts only, one launch each.
template<class Want, class Ghosts>
int launch_pack(Batch& b, Want want, Ghosts ghostsOnly, bool mixed) {
  for (int g = 0; g < 2; ++g) {
    BlockMap bm;
    unsigned grid = 0;
    SPH_TRY(batch_map_items(b, [&](const Problem& p) {
      if (!want(p) || ghostsOnly(p) != (g == 1)) return (int64_t)0;
      if (g == 1) return b.capacityGrids ? p.gcap : p.G;
      return b.capacityGrids ? p.candcap : p.n + p.G; }, 256, &bm, &grid));
    if (!grid) continue;
    if (mixed) pack_mixed_kernel<<<grid, 256, 0, b.stream>>>(b.d_mem, bm, g);
    else pack_records_kernel<<<grid, 256, 0, b.stream>>>(b.d_mem, bm, g);
    batch_count_launch(b);
  }
  return cuda_status(cudaGetLastError(), mixed ? "pack mixed records" : "pack_records");
}

}  // namespace

int pack_records(Batch& b, int need) {
  if (b.memDirty) SPH_TRY(batch_upload(b));
  // which members read the FP64 records before the next pack
  auto wants = [need](const Problem& p) {
    const bool crk = p.prm.hydro == SPHGPU_HYDRO_CRKSPH;
    if (need == PACK_FOR_EVAL)       // grad-h, the FP64 pair loop, the CRKSPH moments
      return crk || p.prm.gradh || p.cfg.precision == SPHGPU_PRECISION_FP64;
    if (need == PACK_FOR_FINALIZE)   // the FP64 summed density, the CRKSPH volumes
      return crk || (p.prm.densityUpdate == SPHGPU_DENSITY_RIGOROUS_SUM &&
                     p.cfg.precision == SPHGPU_PRECISION_FP64);
    return true;
  };
  // internal records the update kernel already wrote (FP64 members)
  auto ghosts = [&](const Problem& p) {
    return need != PACK_ALL && b.packedByUpdate == need && p.cfg.precision == SPHGPU_PRECISION_FP64 &&
           packedByUpdate(p, need);
  };
  return launch_pack(b, wants, ghosts, false);
}

int pack_mixed(Batch& b, bool rigorousSumOnly) {
  if (b.memDirty) SPH_TRY(batch_upload(b));
  const int need = rigorousSumOnly ? PACK_FOR_FINALIZE : PACK_FOR_EVAL;
  auto wants = [&](const Problem& p) {
    return p.cfg.precision == SPHGPU_PRECISION_MIXED && p.prm.hydro == SPHGPU_HYDRO_SPH &&
           (!rigorousSumOnly || p.prm.densityUpdate == SPHGPU_DENSITY_RIGOROUS_SUM);
  };
  auto ghosts = [&](const Problem& p) { return b.packedByUpdate == need && packedByUpdate(p, need); };
  return launch_pack(b, wants, ghosts, true);
}

// ArtificialViscosity::initialize with the Balsara shear correction
// (src/ArtificialViscosity/ArtificialViscosity.cc:123-148): per internal node
// fshear = |div v| / (|div v| + |curl v| + eps^2 max(1e-10, c_s) (det H)^(1/3))
// from the velocity gradient of the last evaluation; ghosts read their root's.
__global__ void __launch_bounds__(256) balsara_kernel(const Member* mem, BlockMap bm) {
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const int64_t n = M.n;
  const int64_t i = mb.block*blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* D = M.D;
  const double* S = M.S;
  double g[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) g[c] = D[(D_DVDX + c)*n + i];
  const double div = fabs(g[0] + g[4] + g[8]);                      // Tensor::Trace
  const double a = g[7] - g[5], b = g[2] - g[6], c = g[3] - g[1];  // zy - yz, xz - zx, yx - xy
  const double curl = sqrt(a*a + b*b + c*c);                        // curlVelocityMagnitude
  const Sym H{S[(S_H + 0)*n + i], S[(S_H + 1)*n + i], S[(S_H + 2)*n + i],
              S[(S_H + 3)*n + i], S[(S_H + 4)*n + i], S[(S_H + 5)*n + i]};
  const double detH = sdet(H);
  const double hmaxinverse = sgn(detH)*pow(fabs(detH), 0.3333333333333333);   // Dim<3>::rootnu
  const double cs = dmax(1.0e-10, S[S_CS*n + i]);                   // negligibleSoundSpeed
  M.fshear[i] = div/(div + curl + M.prm.eps2*cs*hmaxinverse);
}

int launch_balsara(Batch& b) {
  BlockMap bm;
  unsigned grid = 0;
  SPH_TRY(batch_map_items(b, [](const Problem& p) { return p.prm.balsara ? p.n : (int64_t)0; }, 256, &bm, &grid));
  if (grid) { balsara_kernel<<<grid, 256, 0, b.stream>>>(b.d_mem, bm); batch_count_launch(b); }
  return cuda_status(cudaGetLastError(), "balsara");
}

int launch_gradh(Batch& b) {
  BlockMap bm;
  unsigned grid = 0;
  SPH_TRY(batch_map_items(b, [](const Problem& p) { return isSph(p) && p.prm.gradh ? p.n : (int64_t)0; }, 128,
                          &bm, &grid));
  if (grid) { gradh_kernel<<<grid, 128, 0, b.stream>>>(b.d_mem, bm); batch_count_launch(b); }
  return cuda_status(cudaGetLastError(), "gradh");
}

// One launch of the FP64 pair kernel variant <XSPH, TENSILE, COMPAT, BALSARA>.
template<bool X, bool T, bool C, bool B>
void launch_fp64_variant(Batch& b, unsigned grid, BlockMap bm, const Member& one, bool solo) {
  if (solo) sph_eval_fp64_kernel<X, T, C, true, B><<<grid, b.evalThreads, 0, b.stream>>>(b.d_mem, bm, one);
  else sph_eval_fp64_kernel<X, T, C, false, B><<<grid, b.evalThreads, 0, b.stream>>>(b.d_mem, bm, one);
}
using Fp64Launch = void (*)(Batch&, unsigned, BlockMap, const Member&, bool);
// indexed by BALSARA << 3 | XSPH << 2 | TENSILE << 1 | COMPAT
const Fp64Launch kFp64Launch[16] = {
    &launch_fp64_variant<false, false, false, false>, &launch_fp64_variant<false, false, true, false>,
    &launch_fp64_variant<false, true, false, false>, &launch_fp64_variant<false, true, true, false>,
    &launch_fp64_variant<true, false, false, false>, &launch_fp64_variant<true, false, true, false>,
    &launch_fp64_variant<true, true, false, false>, &launch_fp64_variant<true, true, true, false>,
    &launch_fp64_variant<false, false, false, true>, &launch_fp64_variant<false, false, true, true>,
    &launch_fp64_variant<false, true, false, true>, &launch_fp64_variant<false, true, true, true>,
    &launch_fp64_variant<true, false, false, true>, &launch_fp64_variant<true, false, true, true>,
    &launch_fp64_variant<true, true, false, true>, &launch_fp64_variant<true, true, true, true>};

int launch_eval_sph_fp64(Batch& b) {
  auto key = [](const Problem& p) {
    return (p.prm.balsara ? 8 : 0) | (p.prm.XSPH ? 4 : 0) | (p.prm.epsTensile != 0.0 ? 2 : 0) |
           (p.prm.compatible ? 1 : 0);
  };
  const bool solo = b.mem.size() == 1;
  const Member one = solo ? describe_member(*b.mem[0]) : Member{};
  bool present[16] = {};
  for (Problem* p : b.mem) if (isFp64Sph(*p)) present[key(*p)] = true;
  for (int v = 0; v < 16; ++v) {
    if (!present[v]) continue;
    BlockMap bm;
    unsigned grid = 0;
    SPH_TRY(batch_map_items(b, [&](const Problem& p) { return isFp64Sph(p) && key(p) == v ? p.n : (int64_t)0; },
                            b.evalThreads, &bm, &grid));
    if (!grid) continue;
    kFp64Launch[v](b, grid, bm, one, solo);
    batch_count_launch(b);
  }
  return cuda_status(cudaGetLastError(), "evaluate (FP64)");
}

bool summedSph(const Problem& p) { return isSph(p) && p.prm.densityUpdate == SPHGPU_DENSITY_RIGOROUS_SUM; }

int launch_sum_density(Batch& b, bool enforce) {
  BlockMap bm;
  unsigned grid = 0;
  SPH_TRY(batch_map_items(b, [](const Problem& p) {
    return isFp64Sph(p) && summedSph(p) ? p.n : (int64_t)0; }, 128, &bm, &grid));
  if (grid) { sum_density_kernel<<<grid, 128, 0, b.stream>>>(b.d_mem, bm, enforce ? 1 : 0); batch_count_launch(b); }
  return cuda_status(cudaGetLastError(), "sum density");
}

int launch_sum_density_mixed(Batch& b, bool enforce) {
  SPH_TRY(prepare_mixed(b));
  SPH_TRY(pack_mixed(b, true));
  BlockMap bm;
  unsigned grid = 0;
  SPH_TRY(batch_map_items(b, [](const Problem& p) {
    return p.cfg.precision == SPHGPU_PRECISION_MIXED && summedSph(p) ? p.n : (int64_t)0; }, 128, &bm, &grid));
  if (grid) { sum_density_mixed_kernel<<<grid, 128, 0, b.stream>>>(b.d_mem, bm, enforce ? 1 : 0); batch_count_launch(b); }
  return cuda_status(cudaGetLastError(), "sum density (mixed)");
}

int launch_update(Batch& b, double scale, bool timeAdvanceOnly, int mode, int packMode, bool recordMid) {
  if (recordMid && mode == UPDATE_SAVE_START && packMode != PACK_FOR_EVAL) {
    set_error("a record-only mid-point update packs the mid-point records");
    return SPHGPU_ERR_ARG;
  }
  BlockMap bm;
  unsigned grid = 0;
  SPH_TRY(map_nodes(b, 128, &bm, &grid));
  b.packedByUpdate = packMode;
  b.midInS0 = recordMid && mode == UPDATE_SAVE_START;
  const int rm = recordMid ? 1 : 0;
  if (grid) {
    bool compat = false;
    if (!timeAdvanceOnly && mode == UPDATE_FROM_START) for (const Problem* p : b.mem) compat = compat || p->prm.compatible;
    if (compat) update_kernel<true><<<grid, 128, 0, b.stream>>>(b.d_mem, bm, scale, 0, mode, packMode, rm);
    else update_kernel<false><<<grid, 128, 0, b.stream>>>(b.d_mem, bm, scale, timeAdvanceOnly ? 1 : 0, mode, packMode, rm);
    batch_count_launch(b);
  }
  return cuda_status(cudaGetLastError(), "update");
}

int launch_eos(Batch& b) {
  if (b.memDirty) SPH_TRY(batch_upload(b));
  BlockMap bm;
  unsigned grid = 0;
  SPH_TRY(map_nodes(b, 256, &bm, &grid));
  if (grid) { eos_kernel<<<grid, 256, 0, b.stream>>>(b.d_mem, bm); batch_count_launch(b); }
  return cuda_status(cudaGetLastError(), "eos");
}

int launch_enforce_boundaries(Batch& b, bool skipSummed) {
  BlockMap bm;
  unsigned grid = 0;
  SPH_TRY(batch_map_items(b, [&](const Problem& p) { return skipSummed && summedSph(p) ? (int64_t)0 : p.n; },
                          256, &bm, &grid));
  if (grid) { enforce_boundaries_kernel<<<grid, 256, 0, b.stream>>>(b.d_mem, bm); batch_count_launch(b); }
  return cuda_status(cudaGetLastError(), "enforce boundaries");
}

int launch_ideal_h_iteration(Batch& b, double tolerance, double* deltaH) {
  if (b.memDirty) SPH_TRY(batch_upload(b));
  batch_set_scal(b, SC_DELTAH, 0.0);
  BlockMap bm;
  unsigned grid = 0;
  SPH_TRY(map_nodes(b, 128, &bm, &grid));
  if (grid) { ideal_h_iter_kernel<<<grid, 128, 0, b.stream>>>(b.d_mem, bm, tolerance, deltaH); batch_count_launch(b); }
  return cuda_status(cudaGetLastError(), "ideal H iteration");
}

int launch_dt(Batch& b, int slot, bool cachedEig) {
  if (b.memDirty) SPH_TRY(batch_upload(b));
  batch_set_scal(b, slot, kFltMax);
  BlockMap bm;
  unsigned grid = 0;
  SPH_TRY(map_nodes(b, 128, &bm, &grid));
  if (grid) { hydro_dt_kernel<<<grid, 128, 0, b.stream>>>(b.d_mem, bm, slot, cachedEig ? 1 : 0); batch_count_launch(b); }
  return cuda_status(cudaGetLastError(), "dt");
}

int launch_select_dt(Batch& b) {
  SPH_TRY(launch_dt(b, SC_MINDT, true));      // right after the build: H unchanged
  const int nm = (int)b.mem.size();
  select_dt_kernel<<<(nm + 127)/128, 128, 0, b.stream>>>(b.d_mem, nm); batch_count_launch(b);
  return cuda_status(cudaGetLastError(), "select dt");
}

int launch_finish_step(Batch& b) {
  const int nm = (int)b.mem.size();
  finish_step_kernel<<<(nm + 127)/128, 128, 0, b.stream>>>(b.d_mem, nm); batch_count_launch(b);
  return cuda_status(cudaGetLastError(), "finish step");
}

int launch_conservation(Batch& b) {
  if (b.memDirty) SPH_TRY(batch_upload(b));
  std::vector<int64_t> blocks(b.mem.size());
  for (size_t m = 0; m < b.mem.size(); ++m) {
    const int64_t k = (b.mem[m]->n + 255)/256;
    blocks[m] = k < kConsBlocks ? k : kConsBlocks;
  }
  BlockMap bm;
  unsigned grid = 0;
  SPH_TRY(batch_map(b, blocks, &bm, &grid));
  if (grid) { conservation_partials_kernel<<<grid, 256, 0, b.stream>>>(b.d_mem, bm); batch_count_launch(b); }
  const int nm = (int)b.mem.size();
  conservation_final_kernel<<<(nm + 127)/128, 128, 0, b.stream>>>(b.d_mem, nm, bm.first, (int)grid); batch_count_launch(b);
  return cuda_status(cudaGetLastError(), "conservation");
}

int launch_zero_derivs(Batch& b) {
  if (b.memDirty) SPH_TRY(batch_upload(b));
  BlockMap bm;
  unsigned grid = 0;
  SPH_TRY(batch_map_items(b, [](const Problem& p) { return (int64_t)NDERIV*p.n; }, 256, &bm, &grid));
  if (grid) { zero_derivs_kernel<<<grid, 256, 0, b.stream>>>(b.d_mem, bm); batch_count_launch(b); }
  return cuda_status(cudaGetLastError(), "zero derivatives");
}

}  // namespace sphgpu
