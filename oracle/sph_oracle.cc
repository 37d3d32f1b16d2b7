// TEST INFRASTRUCTURE -- the CPU oracle of the SPH hydro path.  Only tests/,
// __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs may
// build, load or call anything in oracle/.  Nothing in the product links it.
//
// A serial FP64 restatement of the reference's SPH fluid path for one
// FluidNodeList in a periodic box, written to follow the reference's loop
// order and expression order (compiled with -O2 -ffp-contract=off, no
// OpenMP: the reference's only OpenMP loop, src/SPH/SPHHydroBase.cc:656-666,
// races on the j-side accumulators and is off in the default build).
//
//   ghosts          PlanarBoundary::setGhostNodes  src/Boundary/PlanarBoundary.cc:114-181
//                   PlanarBoundary::updateGhostNodes :361-395, PeriodicBoundary.cc:87-141
//   violation       PlanarBoundary::setViolationNodes src/Boundary/PlanarBoundary.cc:221-270,
//                   PeriodicBoundary::updateViolationNodes src/Boundary/PeriodicBoundary.cc:171-203
//   connectivity    ConnectivityMap::computeConnectivity src/Neighbor/ConnectivityMap.cc:521-890
//                   (exact predicate :695-718, ascending sort :737), calculatePairInteraction
//                   src/Neighbor/ConnectivityMapInline.hh:169-186 (domain-decomposition
//                   dependent branch)
//   EOS             GammaLawGas::pressure/soundSpeed src/Material/GammaLawGas.cc:166-223
//   Q               MonaghanGingoldViscosity::Piij src/ArtificialViscosity/MonaghanGingoldViscosity.cc:63-133
//                   (Cl/Cq multipliers 1, no Balsara: ArtificialViscosity.cc:99-165)
//   grad-h          computeSPHOmegaGradhCorrection src/SPH/computeSPHOmegaGradhCorrection.cc:28-137
//   derivatives     SPHHydroBase::evaluateDerivatives src/SPH/SPHHydroBase.cc:471-928
//   H               SPHSmoothingScale src/NodeList/SPHSmoothingScale.cc:102-225
//   sum density     computeSPHSumMassDensity src/SPH/computeSPHSumMassDensity.cc:27-111
//   policies        State::update src/DataBase/State.cc:166-287, IncrementFieldList.cc:107-151,
//                   IncrementBoundedState.cc:120-136, ReplaceBoundedState.cc:121-150,
//                   SpecificThermalEnergyPolicy.cc:66-189
//   dt              GenericHydro::dt src/Physics/GenericHydro.cc:114-331,
//                   Integrator::selectDt src/Integrator/Integrator.cc:166-212
//   RK2             CheapSynchronousRK2::step src/Integrator/CheapSynchronousRK2.cc:81-143
//
// Ghost culling (Integrator.cc:494-594) is not applied: culled ghosts are in
// no neighbor list, so culling changes neither neighbor sets nor any sum.

#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <array>
#include <string>
#include <vector>

#include "geom.hh"
#include "table_kernel.hh"
#include "../include/sphgpu.h"

using namespace orc;

namespace {

struct PlanarBC {
  Plane enter, exit;
};

struct Problem {
  sphgpu_config cfg;
  TableKernel W;
  int nInt = 0;
  // Full node arrays: internal [0, nInt) then ghosts.
  std::vector<V3> pos, vel;
  std::vector<double> m, rho, eps, P, cs, omega, eps0;
  std::vector<double> fshear;   // ArtificialViscosity's Balsara shear correction (internal + ghosts)
  std::vector<Sym> H;
  // Ghost bookkeeping, in creation order.
  std::vector<PlanarBC> bcs;                 // 2 per periodic axis, x then y then z
  std::vector<std::vector<int>> control;     // per planar bc: control node indices
  std::vector<std::vector<int>> ghosts;      // per planar bc: ghost node indices
  // Connectivity (internal nodes only), sorted ascending.
  std::vector<std::vector<int>> conn;
  bool haveConn = false;
  // Derivatives (sized to all nodes: the reference's Fields include ghosts).
  std::vector<double> rhoSum, norm, DrhoDt, DepsDt, wns, XSPHw, maxvp, effvp, viscW;
  std::vector<V3> DxDt, DvDt, XSPHdv;
  std::vector<T9> DvDx, localDvDx, M, localM;
  std::vector<Sym> DHDt, Hideal, m2;
  std::vector<std::vector<V3>> pairAcc;
  // CRKSPH (linear order): volume, corrections and their moments (all nodes).
  std::vector<double> vol, A, m0;
  std::vector<V3> B, gradA, m1, gradm0, gradRho;
  std::vector<T9> gradB, gradm1;
  std::vector<T9> qGradVel;   // CRKSPHMonaghanGingoldViscosity::mGradVel (internal + ghosts)
  std::vector<Sym> cm2;                      // CRK second moment (m2 above is the ideal-H one)
  std::vector<std::array<double, 27>> gradm2;
  double time = 0.0, lastDt = 1e-5;
  int cycle = 0;
  bool crkVolumeReady = false;
  std::string err;
};

thread_local std::string g_err;

int numNodes(const Problem& p) { return int(p.pos.size()); }

void resizeAll(Problem& p, int n) {
  p.pos.resize(n); p.vel.resize(n); p.m.resize(n); p.rho.resize(n); p.eps.resize(n);
  p.P.resize(n); p.cs.resize(n); p.omega.resize(n, 1.0); p.eps0.resize(n); p.H.resize(n);
  p.fshear.resize(n, 1.0);
}

// ---------------------------------------------------------------- EOS
double pressureOf(const Problem& p, double rho, double eps) {
  const double g1 = p.cfg.gamma - 1.0;
  const double P = g1*rho*eps;
  // applyPressureLimits with the EquationOfState defaults (no active limits).
  return P < -DBL_MAX ? -DBL_MAX : (P > DBL_MAX ? DBL_MAX : P);
}
double soundSpeedOf(const Problem& p, double rho, double eps) {
  const double g1 = p.cfg.gamma - 1.0;
  return std::sqrt(std::max(0.0, p.cfg.gamma*g1*eps));
}
void updateEOS(Problem& p, int lo, int hi) {
  for (int i = lo; i < hi; ++i) {
    p.P[i] = pressureOf(p, p.rho[i], p.eps[i]);
    p.cs[i] = soundSpeedOf(p, p.rho[i], p.eps[i]);
  }
}

// ---------------------------------------------------------------- boundaries
void makeBoundaries(Problem& p) {
  p.bcs.clear();
  for (int a = 0; a < 3; ++a) {
    if (!p.cfg.periodic[a]) continue;
    V3 n0{0, 0, 0}, n1{0, 0, 0};
    double* c0 = &n0.x; double* c1 = &n1.x;
    c0[a] = 1.0; c1[a] = -1.0;
    const V3 p0{p.cfg.xmin[0], p.cfg.xmin[1], p.cfg.xmin[2]};
    const V3 p1{p.cfg.xmax[0], p.cfg.xmax[1], p.cfg.xmax[2]};
    const Plane plane1(p0, n0), plane2(p1, n1);
    // PeriodicBoundary(plane1, plane2): mPlane1Boundary(plane1, plane2),
    // mPlane2Boundary(plane2, plane1); PlanarBoundary(enter, exit).
    p.bcs.push_back(PlanarBC{plane1, plane2});
    p.bcs.push_back(PlanarBC{plane2, plane1});
  }
}

// Copy every field from control to ghost for one planar boundary (applyGhostBoundary).
void copyGhostFields(Problem& p, int b) {
  const auto& c = p.control[b];
  const auto& g = p.ghosts[b];
  for (size_t k = 0; k < c.size(); ++k) {
    const int s = c[k], d = g[k];
    p.vel[d] = p.vel[s]; p.m[d] = p.m[s]; p.rho[d] = p.rho[s]; p.eps[d] = p.eps[s];
    p.P[d] = p.P[s]; p.cs[d] = p.cs[s]; p.omega[d] = p.omega[s]; p.eps0[d] = p.eps0[s];
  }
}

// updateGhostNodes: positions mapped through the planes, H copied.
void updateGhostNodes(Problem& p, int b) {
  const auto& c = p.control[b];
  const auto& g = p.ghosts[b];
  for (size_t k = 0; k < c.size(); ++k) {
    // mapPosition(pos, mExitPlane, mEnterPlane)
    p.pos[g[k]] = mapPositionThroughPlanes(p.pos[c[k]], p.bcs[b].exit, p.bcs[b].enter);
    p.H[g[k]] = p.H[c[k]];
  }
}

void setGhostNodes(Problem& p) {
  resizeAll(p, p.nInt);
  p.control.assign(p.bcs.size(), {});
  p.ghosts.assign(p.bcs.size(), {});
  const double kernelExtent = p.W.extent;
  for (size_t b = 0; b < p.bcs.size(); ++b) {
    const PlanarBC& bc = p.bcs[b];
    const int n = numNodes(p);
    double hmax = 0.0;
    for (int i = 0; i != n; ++i) {
      const double hmaxi = 1.0/minElement(eigenValues(p.H[i]));
      if (hmaxi > hmax && std::min(bc.exit.minimumDistance(p.pos[i]), bc.enter.minimumDistance(p.pos[i])) < kernelExtent*hmaxi)
        hmax = hmaxi;
    }
    std::vector<int>& ctrl = p.control[b];
    if (hmax > 0.0) {
      for (int i = 0; i != n; ++i) {
        const double disti = bc.exit.signedDistance(p.pos[i])/hmax;
        if (disti >= 0.0 && disti <= kernelExtent) ctrl.push_back(i);
      }
    }
    resizeAll(p, n + int(ctrl.size()));
    for (size_t k = 0; k < ctrl.size(); ++k) p.ghosts[b].push_back(n + int(k));
    updateGhostNodes(p, b);
  }
}

// Integrator::applyGhostBoundaries: update ghost positions/H, then every state field.
void applyGhostBoundaries(Problem& p) {
  for (size_t b = 0; b < p.bcs.size(); ++b) updateGhostNodes(p, b);
  for (size_t b = 0; b < p.bcs.size(); ++b) copyGhostFields(p, b);
}

// Integrator::setViolationNodes for the periodic boundaries (positions only;
// every other field travels with the node).
void enforceBoundaries(Problem& p) {
  for (size_t pb = 0; pb + 1 < p.bcs.size(); pb += 2) {
    for (int sub = 0; sub < 2; ++sub) {
      const PlanarBC& bc = p.bcs[pb + sub];
      for (int i = 0; i < p.nInt; ++i) {
        if (bc.enter.compare(p.pos[i]) == 1) p.pos[i] = mapPositionThroughPlanes(p.pos[i], bc.enter, bc.exit);
      }
    }
    // PeriodicBoundary::updateViolationNodes multi-wrap fix for the union of
    // the two violation lists.
    const Plane& plane1 = p.bcs[pb].enter;
    const Plane& plane2 = p.bcs[pb].exit;
    const V3 origin = plane1.point, nhat = plane1.normal;
    const double L = plane1.minimumDistance(plane2.point);
    for (int i = 0; i < p.nInt; ++i) {
      if (plane1.compare(p.pos[i]) == 1 || plane2.compare(p.pos[i]) == 1) {
        const V3 p0 = vadd(p.pos[i], vmul(nhat, dot(vsub(origin, p.pos[i]), nhat)));
        const double f = std::max(-1.0, std::min(1.0, std::fmod(plane1.signedDistance(p.pos[i])/L, 1.0)));
        p.pos[i] = vadd(p0, vmul(nhat, f*L));
      }
    }
  }
}

// ---------------------------------------------------------------- connectivity
void computeConnectivity(Problem& p) {
  const int n = numNodes(p);
  const double kernelExtent = p.W.extent;
  const double kernelExtent2 = kernelExtent*kernelExtent;
  // Superset generator: uniform cells of size >= kernelExtent * max h.
  double hmax = 0.0;
  V3 lo{DBL_MAX, DBL_MAX, DBL_MAX}, hi{-DBL_MAX, -DBL_MAX, -DBL_MAX};
  for (int i = 0; i < n; ++i) {
    hmax = std::max(hmax, 1.0/minElement(eigenValues(p.H[i])));
    lo.x = std::min(lo.x, p.pos[i].x); lo.y = std::min(lo.y, p.pos[i].y); lo.z = std::min(lo.z, p.pos[i].z);
    hi.x = std::max(hi.x, p.pos[i].x); hi.y = std::max(hi.y, p.pos[i].y); hi.z = std::max(hi.z, p.pos[i].z);
  }
  const double cell = kernelExtent*hmax*1.01 + 1e-300;
  const int nx = std::max(1, int((hi.x - lo.x)/cell) + 1);
  const int ny = std::max(1, int((hi.y - lo.y)/cell) + 1);
  const int nz = std::max(1, int((hi.z - lo.z)/cell) + 1);
  std::vector<std::vector<int>> cells(size_t(nx)*ny*nz);
  auto cidx = [&](const V3& r, int& cx, int& cy, int& cz) {
    cx = std::min(nx - 1, std::max(0, int((r.x - lo.x)/cell)));
    cy = std::min(ny - 1, std::max(0, int((r.y - lo.y)/cell)));
    cz = std::min(nz - 1, std::max(0, int((r.z - lo.z)/cell)));
  };
  for (int i = 0; i < n; ++i) {
    int cx, cy, cz; cidx(p.pos[i], cx, cy, cz);
    cells[(size_t(cz)*ny + cy)*nx + cx].push_back(i);
  }
  p.conn.assign(p.nInt, {});
  for (int i = 0; i < p.nInt; ++i) {
    const V3& ri = p.pos[i];
    const Sym& Hi = p.H[i];
    int cx, cy, cz; cidx(ri, cx, cy, cz);
    std::vector<int>& nb = p.conn[i];
    for (int dz = -1; dz <= 1; ++dz) for (int dy = -1; dy <= 1; ++dy) for (int dx = -1; dx <= 1; ++dx) {
      const int x = cx + dx, y = cy + dy, z = cz + dz;
      if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) continue;
      for (int j : cells[(size_t(z)*ny + y)*nx + x]) {
        const V3 rij = vsub(ri, p.pos[j]);
        const double eta2i = mag2(sdot(Hi, rij));
        const double eta2j = mag2(sdot(p.H[j], rij));
        if (eta2i <= kernelExtent2 || eta2j <= kernelExtent2) {
          if (i != j) nb.push_back(j);
        }
      }
    }
    std::sort(nb.begin(), nb.end());
  }
  p.haveConn = true;
}

// calculatePairInteraction for one NodeList: j > i (ghosts have j >= nInt > i).
inline bool calcPair(int i, int j) { return j > i; }

// ---------------------------------------------------------------- physics
void zeroDerivs(Problem& p) {
  const int n = numNodes(p);
  p.rhoSum.assign(n, 0.0); p.norm.assign(n, 0.0); p.DrhoDt.assign(n, 0.0); p.DepsDt.assign(n, 0.0);
  p.wns.assign(n, 0.0); p.XSPHw.assign(n, 0.0); p.maxvp.assign(n, 0.0); p.effvp.assign(n, 0.0);
  p.viscW.assign(n, 0.0);
  p.DxDt.assign(n, V3{0, 0, 0}); p.DvDt.assign(n, V3{0, 0, 0}); p.XSPHdv.assign(n, V3{0, 0, 0});
  p.DvDx.assign(n, tzero()); p.localDvDx.assign(n, tzero()); p.M.assign(n, tzero()); p.localM.assign(n, tzero());
  p.DHDt.assign(n, Sym{0, 0, 0, 0, 0, 0}); p.Hideal.assign(n, Sym{0, 0, 0, 0, 0, 0}); p.m2.assign(n, Sym{0, 0, 0, 0, 0, 0});
  p.pairAcc.assign(n, {});
}

void gradhCorrection(Problem& p) {
  const int n = numNodes(p);
  std::vector<double> gradsum(n, 0.0);
  for (int i = 0; i < n; ++i) p.omega[i] = 0.0;
  for (int i = 0; i < p.nInt; ++i) {
    if (p.conn[i].empty()) { p.omega[i] = 1.0; continue; }
    const V3& ri = p.pos[i];
    const Sym& Hi = p.H[i];
    const double Hdeti = sdet(Hi);
    const double W0 = p.W.kernelValue(0.0, Hdeti);
    p.omega[i] += W0;
    for (int j : p.conn[i]) {
      if (!calcPair(i, j)) continue;
      const Sym& Hj = p.H[j];
      const double Hdetj = sdet(Hj);
      const V3 rij = vsub(ri, p.pos[j]);
      const double etai = mag(sdot(Hi, rij));
      const double etaj = mag(sdot(Hj, rij));
      const auto WWi = p.W.kernelAndGradValue(etai, Hdeti);
      const auto WWj = p.W.kernelAndGradValue(etaj, Hdetj);
      p.omega[i] += WWi.first;
      gradsum[i] += etai*WWi.second;
      p.omega[j] += WWj.first;
      gradsum[j] += etaj*WWj.second;
    }
    p.omega[i] = -gradsum[i]/(3*p.omega[i]);
  }
}

// MonaghanGingoldViscosity::Piij, returning the diagonal value e/rho of each side.
// fsi, fsj: the two nodes' shear corrections (ArtificialViscosity.cc:123-148; 1 without it).
inline void Piij(const Problem& p, const V3& etai, const V3& vi, double rhoi, double csi,
                 const V3& etaj, const V3& vj, double rhoj, double csj, T9& QPi, T9& QPj,
                 double fsi = 1.0, double fsj = 1.0) {
  double Cl = p.cfg.Cl, Cq = p.cfg.Cq;
  const double eps2 = p.cfg.epsilon2;
  const double fCli = 1.0, fCqi = 1.0, fClj = 1.0, fCqj = 1.0;
  const double fshear = std::max(fsi, fsj);
  Cl *= 0.5*(fCli + fClj)*fshear;
  Cq *= 0.5*(fCqi + fCqj)*fshear;
  const V3 vij = vsub(vi, vj);
  const double mui = dot(vij, etai)/(mag2(etai) + eps2);
  const double muj = dot(vij, etaj)/(mag2(etaj) + eps2);
  const bool lin = p.cfg.linearInExpansion != 0, quad = p.cfg.quadraticInExpansion != 0;
  const double mi0 = std::min(0.0, mui), mj0 = std::min(0.0, muj);
  const double ei = -Cl*csi*(lin ? mui : mi0) + Cq*(quad ? -sgn(mui)*mui*mui : mi0*mi0);
  const double ej = -Cl*csj*(lin ? muj : mj0) + Cq*(quad ? -sgn(muj)*muj*muj : mj0*mj0);
  QPi = tdiag(ei/rhoi);
  QPj = tdiag(ej/rhoj);
}

void evaluateDerivatives(Problem& p) {
  zeroDerivs(p);
  const TableKernel& W = p.W;
  const TableKernel& WQ = p.W;
  const double tiny = 1.0e-30;
  const double W0 = W.kernelValue(0.0, 1.0);
  const double nPerh = p.cfg.nPerh;
  const double WnPerh = W.kernelValue(1.0/nPerh, 1.0);
  const bool compatible = p.cfg.compatibleEnergyEvolution != 0;
  const bool XSPH = p.cfg.XSPH != 0;
  for (int i = 0; i < p.nInt; ++i) {
    const V3& ri = p.pos[i]; const double mi = p.m[i]; const V3& vi = p.vel[i];
    const double rhoi = p.rho[i]; const double Pi = p.P[i]; const Sym& Hi = p.H[i];
    const double ci = p.cs[i]; const double omegai = p.omega[i];
    const double Hdeti = sdet(Hi);
    const double safeOmegai = safeInv(omegai, tiny);
    double maxvp = p.maxvp[i];
    for (int j : p.conn[i]) {
      if (!calcPair(i, j)) continue;
      const V3& rj = p.pos[j]; const double mj = p.m[j]; const V3& vj = p.vel[j];
      const double rhoj = p.rho[j]; const double Pj = p.P[j]; const Sym& Hj = p.H[j];
      const double cj = p.cs[j]; const double omegaj = p.omega[j];
      const double Hdetj = sdet(Hj);
      const double safeOmegaj = safeInv(omegaj, tiny);
      const bool sameMatij = true;

      const V3 rij = vsub(ri, rj);
      const V3 etai = sdot(Hi, rij);
      const V3 etaj = sdot(Hj, rij);
      const double etaMagi = mag(etai);
      const double etaMagj = mag(etaj);

      const V3 Hetai = sdot(Hi, unitVector(etai));
      const auto WWi = W.kernelAndGradValue(etaMagi, Hdeti);
      const double Wi = WWi.first, gWi = WWi.second;
      const V3 gradWi = vmul(Hetai, gWi);
      const V3 gradWQi = vmul(Hetai, WQ.gradValue(etaMagi, Hdeti));

      const V3 Hetaj = sdot(Hj, unitVector(etaj));
      const auto WWj = W.kernelAndGradValue(etaMagj, Hdetj);
      const double Wj = WWj.first, gWj = WWj.second;
      const V3 gradWj = vmul(Hetaj, gWj);
      const V3 gradWQj = vmul(Hetaj, WQ.gradValue(etaMagj, Hdetj));

      const double fweightij = sameMatij ? 1.0 : mj*rhoi/(mi*rhoj);
      const double rij2 = mag2(rij);
      const Sym thpt = smul(selfdyad(rij), safeInvVar(rij2*rij2*rij2));
      p.wns[i] += fweightij*std::abs(gWi);
      p.wns[j] += 1.0/fweightij*std::abs(gWj);
      p.m2[i] = sadd(p.m2[i], smul(thpt, fweightij*mag2(gradWi)));
      p.m2[j] = sadd(p.m2[j], smul(thpt, 1.0/fweightij*mag2(gradWj)));

      p.rhoSum[i] += mj*Wi;
      p.rhoSum[j] += mi*Wj;
      p.norm[i] += mi/rhoi*Wi;
      p.norm[j] += mj/rhoj*Wj;

      const V3 vij = vsub(vi, vj);
      T9 QPi, QPj;
      Piij(p, etai, vi, rhoi, ci, etaj, vj, rhoj, cj, QPi, QPj, p.fshear[i], p.fshear[j]);
      const V3 Qacci = vmul(tvdot(QPi, gradWQi), 0.5);
      const V3 Qaccj = vmul(tvdot(QPj, gradWQj), 0.5);
      const double workQi = dot(vij, Qacci);
      const double workQj = dot(vij, Qaccj);
      const double Qi = rhoi*rhoi*(maxAbsElement(V3{QPi.xx, QPi.yy, QPi.zz}));
      const double Qj = rhoj*rhoj*(maxAbsElement(V3{QPj.xx, QPj.yy, QPj.zz}));
      maxvp = std::max(maxvp, Qi);
      p.maxvp[j] = std::max(p.maxvp[j], Qj);
      p.effvp[i] += mj/rhoj*Qi*Wi;
      p.effvp[j] += mi/rhoi*Qj*Wj;
      p.viscW[i] += mj*workQi;
      p.viscW[j] += mi*workQj;

      const double fij = p.cfg.epsTensile*pow4(Wi/(Hdeti*WnPerh));
      const double Ri = fij*(Pi < 0.0 ? -Pi : 0.0);
      const double Rj = fij*(Pj < 0.0 ? -Pj : 0.0);
      const double Peffi = Pi + Ri;
      const double Peffj = Pj + Rj;

      const double Prhoi = safeOmegai*Peffi/(rhoi*rhoi);
      const double Prhoj = safeOmegaj*Peffj/(rhoj*rhoj);
      const V3 deltaDvDt = vadd(vadd(vadd(vmul(gradWi, Prhoi), vmul(gradWj, Prhoj)), Qacci), Qaccj);
      p.DvDt[i] = vadd(p.DvDt[i], vmul(deltaDvDt, -mj));
      p.DvDt[j] = vadd(p.DvDt[j], vmul(deltaDvDt, mi));

      p.DepsDt[i] += mj*(Prhoi*dot(vij, gradWi) + workQi);
      p.DepsDt[j] += mi*(Prhoj*dot(vij, gradWj) + workQj);
      if (compatible) {
        p.pairAcc[i].push_back(vmul(deltaDvDt, -mj));
        p.pairAcc[j].push_back(vmul(deltaDvDt, mi));
      }

      const T9 deltaDvDxi = tmul(dyad(vij, gradWi), mj);
      const T9 deltaDvDxj = tmul(dyad(vij, gradWj), mi);
      taddto(p.DvDx[i], tneg(deltaDvDxi));
      tsubfrom(p.DvDx[j], deltaDvDxj);
      if (sameMatij) {
        taddto(p.localDvDx[i], tneg(deltaDvDxi));
        tsubfrom(p.localDvDx[j], deltaDvDxj);
      }

      if (XSPH && sameMatij) {
        const double wXSPHij = 0.5*(mi/rhoi*Wi + mj/rhoj*Wj);
        p.XSPHw[i] += wXSPHij;
        p.XSPHw[j] += wXSPHij;
        p.XSPHdv[i] = vsub(p.XSPHdv[i], vmul(vij, wXSPHij));
        p.XSPHdv[j] = vadd(p.XSPHdv[j], vmul(vij, wXSPHij));
      }

      taddto(p.M[i], tmul(dyad(rij, gradWi), -mj));
      tsubfrom(p.M[j], tmul(dyad(rij, gradWj), mi));
      if (sameMatij) {
        taddto(p.localM[i], tmul(dyad(rij, gradWi), -mj));
        tsubfrom(p.localM[j], tmul(dyad(rij, gradWj), mi));
      }
    }
    p.maxvp[i] = std::max(p.maxvp[i], maxvp);

    const int numNeighborsi = int(p.conn[i].size());
    p.rhoSum[i] += mi*W0*Hdeti;
    p.norm[i] += mi/rhoi*W0*Hdeti;

    T9& Mi = p.M[i]; T9& DvDxi = p.DvDx[i];
    if (p.cfg.correctVelocityGradient && std::abs(tdet(Mi)) > 1.0e-10 && numNeighborsi > 8) {
      Mi = tinverse(Mi);
      DvDxi = tdot(DvDxi, Mi);
    } else {
      DvDxi = tdiv(DvDxi, rhoi);
    }
    T9& localMi = p.localM[i]; T9& localDvDxi = p.localDvDx[i];
    if (p.cfg.correctVelocityGradient && std::abs(tdet(localMi)) > 1.0e-10 && numNeighborsi > 8) {
      localMi = tinverse(localMi);
      localDvDxi = tdot(localDvDxi, localMi);
    } else {
      localDvDxi = tdiv(localDvDxi, rhoi);
    }

    p.DrhoDt[i] = -rhoi*ttrace(DvDxi);

    p.wns[i] = CubeRootHalley2(std::max(0.0, p.wns[i]/Hdeti));
    p.m2[i] = sdiv(p.m2[i], Hdeti*Hdeti);

    if (XSPH) {
      p.XSPHw[i] += Hdeti*mi/rhoi*W0;
      p.DxDt[i] = vadd(vi, vdiv(p.XSPHdv[i], std::max(tiny, p.XSPHw[i])));
    } else {
      p.DxDt[i] = vi;
    }

    // SPHSmoothingScale::smoothingScaleDerivative
    p.DHDt[i] = smul(sdiv(sneg(Hi), 3), ttrace(DvDxi));
    // SPHSmoothingScale::idealSmoothingScale (n0 count is unused by the result)
    const double zerothMoment = p.wns[i];
    double currentNodesPerSmoothingScale;
    if (fuzzyEqual(zerothMoment, 0.0)) currentNodesPerSmoothingScale = 0.5*nPerh;
    else currentNodesPerSmoothingScale = W.equivalentNodesPerSmoothingScale(zerothMoment);
    const double s = std::min(4.0, std::max(0.25, nPerh/(currentNodesPerSmoothingScale + 1.0e-30)));
    double a;
    if (s < 1.0) a = 0.4*(1.0 + s*s);
    else a = 0.4*(1.0 + 1.0/(s*s*s));
    const double hi0 = 1.0/Hi.xx;
    const double hi1 = std::min(p.cfg.hmax, std::max(p.cfg.hmin, hi0*(1.0 - a + a*s)));
    const double inv = 1.0/hi1;
    p.Hideal[i] = Sym{1.0*inv, 0.0*inv, 0.0*inv, 1.0*inv, 0.0*inv, 1.0*inv};
  }
}

// finalizeDerivatives (compatible energy): ghost copies of DvDt and DepsDt.
void finalizeDerivatives(Problem& p) {
  if (!p.cfg.compatibleEnergyEvolution) return;
  for (size_t b = 0; b < p.bcs.size(); ++b) {
    for (size_t k = 0; k < p.control[b].size(); ++k) {
      const int s = p.control[b][k], d = p.ghosts[b][k];
      p.DvDt[d] = p.DvDt[s];
      p.DepsDt[d] = p.DepsDt[s];
    }
  }
}

void computeSumMassDensity(Problem& p) {
  const int n = numNodes(p);
  for (int i = 0; i < n; ++i) p.rho[i] = 0.0;
  for (int i = 0; i < p.nInt; ++i) {
    const V3& ri = p.pos[i]; const double mi = p.m[i]; const Sym& Hi = p.H[i];
    const double Hdeti = sdet(Hi);
    const double W0 = p.W.kernelValue(0.0, Hdeti);
    p.rho[i] += mi*W0;
    for (int j : p.conn[i]) {
      if (!calcPair(i, j)) continue;
      const V3& rj = p.pos[j]; const double mj = p.m[j]; const Sym& Hj = p.H[j];
      const double Hdetj = sdet(Hj);
      const V3 rij = vsub(ri, rj);
      const double etai = mag(sdot(Hi, rij));
      const double etaj = mag(sdot(Hj, rij));
      const double Wi = p.W.kernelValue(etai, Hdeti);
      const double Wj = p.W.kernelValue(etaj, Hdetj);
      p.rho[i] += mj*Wj;
      p.rho[j] += mi*Wi;
    }
  }
}

// IncrementBoundedState / ReplaceBoundedState<SymTensor> for H
// (src/DataBase/IncrementBoundedState.cc:131-133, ReplaceBoundedState.cc:134-136):
// min(1/hmin, max(1/hmax, H)) with the eigenvalue limiters; SPHHydroBase
// registers the policy with 1/hmax and 1/hmin (src/SPH/SPHHydroBase.cc:290-296).
Sym boundH(const Problem& p, const Sym& H) {
  const double hmaxInv = 1.0/p.cfg.hmax, hminInv = 1.0/p.cfg.hmin;
  return symMin(hminInv, symMax(hmaxInv, H));
}

// State::update for the SPH policies.  timeAdvanceOnly selects updateAsIncrement.
bool stateUpdate(Problem& p, double multiplier, bool timeAdvanceOnly) {
  const int n = p.nInt;
  // Pass 1 (no dependencies, key order): H, mass density, position, specific thermal energy.
  for (int i = 0; i < n; ++i) {
    Sym Hn;
    if (p.cfg.HUpdate == SPHGPU_H_INTEGRATE || timeAdvanceOnly) {
      Hn = sadd(p.H[i], smul(p.DHDt[i], multiplier));
    } else {
      Hn = p.Hideal[i];
    }
    p.H[i] = boundH(p, Hn);
  }
  if (p.cfg.densityUpdate == SPHGPU_DENSITY_INTEGRATE || true) {
    for (int i = 0; i < n; ++i)
      p.rho[i] = std::min(p.cfg.rhoMax, std::max(p.cfg.rhoMin, p.rho[i] + multiplier*(p.DrhoDt[i])));
  }
  for (int i = 0; i < n; ++i) p.pos[i] = vadd(p.pos[i], vmul(p.DxDt[i], multiplier));
  if (p.cfg.compatibleEnergyEvolution && !timeAdvanceOnly) {
    // SpecificThermalEnergyPolicy::update
    const int nn = numNodes(p);
    std::vector<double> DepsDt(nn, 0.0);
    std::vector<int> offset(nn, 0);
    const double hdt = 0.5*multiplier;
    const double epsilon = 2.220446049250313e-16;
    for (int i = 0; i < n; ++i) {
      const double weighti = std::abs(p.DepsDt[i]) + epsilon;
      const double mi = p.m[i];
      const V3& vi = p.vel[i];
      const V3& ai = p.DvDt[i];
      const V3 vi12 = vadd(vi, vmul(ai, hdt));
      for (int j : p.conn[i]) {
        if (!calcPair(i, j)) continue;
        const double weightj = std::abs(p.DepsDt[j]) + epsilon;
        const double mj = p.m[j];
        const V3& vj = p.vel[j];
        const V3& aj = p.DvDt[j];
        const V3 vj12 = vadd(vj, vmul(aj, hdt));
        const V3 vji12 = vsub(vj12, vi12);
        const V3& pai = p.pairAcc[i][offset[i]++];
        offset[j]++;
        const double duij = dot(vji12, pai);
        const double wi = weighti/(weighti + weightj);
        DepsDt[i] += wi*duij;
        DepsDt[j] += (1.0 - wi)*duij*mi/mj;
      }
      p.eps[i] += DepsDt[i]*multiplier;
    }
  } else {
    for (int i = 0; i < n; ++i) p.eps[i] += multiplier*(p.DepsDt[i]);
  }
  // Pass 2: pressure, sound speed, velocity.
  updateEOS(p, 0, n);
  for (int i = 0; i < n; ++i) p.vel[i] = vadd(p.vel[i], vmul(p.DvDt[i], multiplier));
  return true;
}

double hydroDt(const Problem& p) {
  double minDt = FLT_MAX;
  const double nPerh = p.cfg.nPerh;
  for (int i = 0; i < p.nInt; ++i) {
    const double nodeScale = 1.0/maxElement(eigenValues(p.H[i]))/nPerh;
    const double csDt = nodeScale/(p.cs[i] + FLT_MIN);
    if (csDt < minDt) minDt = csDt;
    const double csq = std::sqrt(p.maxvp[i]/p.rho[i]);
    const double csqDt = nodeScale/(csq + FLT_MIN);
    if (csqDt < minDt) minDt = csqDt;
    const double divVelocity = ttrace(p.DvDx[i]);
    const double divvDt = 1.0/(std::abs(divVelocity) + FLT_MIN);
    if (divvDt < minDt) minDt = divvDt;
    const V3& vi = p.vel[i];
    for (int j : p.conn[i]) {
      const double vij = mag(vsub(vi, p.vel[j]));
      const double dtVelDiff = nodeScale*safeInvVar(vij, 1e-30);
      if (dtVelDiff < minDt) minDt = dtVelDiff;
    }
    const double dtAcc = std::sqrt(nodeScale/(mag(p.DvDt[i]) + FLT_MIN));
    if (dtAcc < minDt) minDt = dtAcc;
    if (p.cfg.useVelocityMagnitudeForDt) {
      const double velDt = nodeScale/(mag(vi) + 1.0e-10);
      if (velDt < minDt) minDt = velDt;
    }
  }
  return p.cfg.cfl*minDt;
}

double selectDt(Problem& p) {
  const double dtMin = p.cfg.dtMin, dtMax = p.cfg.dtMax;
  double dt = dtMax;
  const double vote = hydroDt(p);
  if (vote > 0.0 && vote < dt) dt = vote;
  dt = std::min(dt, p.cfg.dtGrowth*p.lastDt);
  dt = std::min(dtMax, std::max(dtMin, dt));
  return dt;
}

// ArtificialViscosity::initialize with the Balsara shear correction
// (src/ArtificialViscosity/ArtificialViscosity.cc:123-148): from the velocity
// gradient of the last evaluation, the derivatives not yet zeroed; ghosts
// take their control node's value (applyFieldListGhostBoundary).
void balsaraShearCorrection(Problem& p) {
  for (int i = 0; i < p.nInt; ++i) {
    const T9 g = i < int(p.DvDx.size()) ? p.DvDx[i] : tzero();   // none before the first evaluation
    const double div = std::abs(g.xx + g.yy + g.zz);
    const double a = g.zy - g.yz, b = g.xz - g.zx, c = g.yx - g.xy;
    const double curl = std::sqrt(a*a + b*b + c*c);
    const double hmaxinverse = CubeRootHalley2(sdet(p.H[i]));
    const double cs = std::max(1.0e-10, p.cs[i]);
    p.fshear[i] = div/(div + curl + p.cfg.epsilon2*cs*hmaxinverse);
  }
  for (size_t b = 0; b < p.bcs.size(); ++b)
    for (size_t k = 0; k < p.control[b].size(); ++k) p.fshear[p.ghosts[b][k]] = p.fshear[p.control[b][k]];
}

void initializeDerivatives(Problem& p) {
  if (p.cfg.balsaraShearCorrection) balsaraShearCorrection(p);
  if (p.cfg.gradhCorrection) {
    gradhCorrection(p);
    for (size_t b = 0; b < p.bcs.size(); ++b)
      for (size_t k = 0; k < p.control[b].size(); ++k) p.omega[p.ghosts[b][k]] = p.omega[p.control[b][k]];
  }
}

void finalizeStep(Problem& p) {
  if (p.cfg.densityUpdate == SPHGPU_DENSITY_RIGOROUS_SUM) computeSumMassDensity(p);
}

// Integrator::preStepInitialize with the default boundary cadence: ghosts and
// connectivity rebuilt every cycle, then ghost state refreshed.
void preStepInitialize(Problem& p) {
  setGhostNodes(p);
  computeConnectivity(p);
  applyGhostBoundaries(p);
}

bool stepRK2(Problem& p, double& dtOut) {
  const double t = p.time;
  preStepInitialize(p);
  for (int i = 0; i < numNodes(p); ++i) p.eps0[i] = p.eps[i];
  const double dt = selectDt(p);
  const double hdt = 0.5*dt;
  // state0 copy (all nodes, ghosts included)
  const std::vector<V3> pos0 = p.pos, vel0 = p.vel;
  const std::vector<double> rho0 = p.rho, eps0 = p.eps, P0 = p.P, cs0 = p.cs, om0 = p.omega;
  const std::vector<Sym> H0 = p.H;
  if (!stateUpdate(p, hdt, true)) return false;
  p.time = t + hdt;
  applyGhostBoundaries(p);
  initializeDerivatives(p);
  evaluateDerivatives(p);
  finalizeDerivatives(p);
  p.pos = pos0; p.vel = vel0; p.rho = rho0; p.eps = eps0; p.P = P0; p.cs = cs0; p.omega = om0; p.H = H0;
  if (!stateUpdate(p, dt, false)) return false;
  p.time = t + dt;
  applyGhostBoundaries(p);
  finalizeStep(p);
  enforceBoundaries(p);
  p.cycle += 1;
  p.time = t + dt;
  p.lastDt = dt;
  dtOut = dt;
  return true;
}

// ====================================================================== CRKSPH
//   moments      computeCRKSPHMoments src/CRKSPH/computeCRKSPHMoments.cc:40-287 (LinearOrder,
//                NodeCoupling = 1)
//   corrections  computeLinearCRKSPHCorrections src/CRKSPH/computeCRKSPHCorrections.cc:210-283
//   kernel       CRKSPHKernelAndGradient src/CRKSPH/CRKSPHUtilitiesInline.hh:58-129
//   derivatives  CRKSPHHydroBase::evaluateDerivatives src/CRKSPH/CRKSPHHydroBase.cc:646-1102
//   volume       computeCRKSPHSumVolume src/CRKSPH/computeCRKSPHSumVolume.cc:43-127,
//                ContinuityVolumePolicy::update src/CRKSPH/ContinuityVolumePolicy.cc:67-95
//   density      computeCRKSPHSumMassDensity src/CRKSPH/computeCRKSPHSumMassDensity.cc:28-139

inline double& el(V3& v, int i) { return (&v.x)[i]; }
inline double el(const V3& v, int i) { return (&v.x)[i]; }
inline double& el(T9& t, int i, int j) { return (&t.xx)[3*i + j]; }
inline double el(const T9& t, int i, int j) { return (&t.xx)[3*i + j]; }
inline double& sel(Sym& s, int i, int j) {
  static const int map[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
  return (&s.xx)[map[i][j]];
}
inline double sel(const Sym& s, int i, int j) {
  static const int map[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
  return (&s.xx)[map[i][j]];
}

template<typename T>
void ghostCopy(Problem& p, std::vector<T>& f) {
  for (size_t b = 0; b < p.bcs.size(); ++b)
    for (size_t k = 0; k < p.control[b].size(); ++k) f[p.ghosts[b][k]] = f[p.control[b][k]];
}

void crkResize(Problem& p) {
  const int n = numNodes(p);
  p.vol.resize(n, 0.0); p.A.resize(n, 0.0); p.B.resize(n, V3{0, 0, 0});
  p.gradA.resize(n, V3{0, 0, 0}); p.gradB.resize(n, tzero());
}

void crkSumVolume(Problem& p) {
  const int n = numNodes(p);
  const double etaVolMax = (0.5*p.W.extent)*(0.5*p.W.extent)*(0.5*p.W.extent)*(4.0/3.0*M_PI);
  p.vol.assign(n, 0.0);
  for (int i = 0; i < p.nInt; ++i) {
    const V3& ri = p.pos[i];
    const Sym& Hi = p.H[i];
    const double Hdeti = sdet(Hi);
    for (int j : p.conn[i]) {
      if (!calcPair(i, j)) continue;
      const Sym& Hj = p.H[j];
      const double Hdetj = sdet(Hj);
      const V3 rij = vsub(ri, p.pos[j]);
      const double etai = mag(sdot(Hi, rij));
      const double etaj = mag(sdot(Hj, rij));
      p.vol[i] += p.W.kernelValue(etai, Hdeti);
      p.vol[j] += p.W.kernelValue(etaj, Hdetj);
    }
    p.vol[i] += p.W.kernelValue(0.0, Hdeti);
    p.vol[i] = std::min(etaVolMax/Hdeti, 1.0/p.vol[i]);
  }
  ghostCopy(p, p.vol);
}

void crkSumDensity(Problem& p) {
  const int n = numNodes(p);
  std::vector<double> wsum(n, 0.0), vol1(n, 0.0);
  for (int i = 0; i < n; ++i) p.rho[i] = 0.0;
  for (int i = 0; i < p.nInt; ++i) {
    const V3& ri = p.pos[i];
    const double mi = p.m[i], Vi = p.vol[i];
    const Sym& Hi = p.H[i];
    const double Hdeti = sdet(Hi);
    for (int j : p.conn[i]) {
      if (!calcPair(i, j)) continue;
      const double mj = p.m[j], Vj = p.vol[j];
      const Sym& Hj = p.H[j];
      const double Hdetj = sdet(Hj);
      const V3 rij = vsub(ri, p.pos[j]);
      const double Wi = p.W.kernelValue(mag(sdot(Hi, rij)), Hdeti);
      const double Wj = p.W.kernelValue(mag(sdot(Hj, rij)), Hdetj);
      wsum[i] += Vj*Wj;
      wsum[j] += Vi*Wi;
      p.rho[i] += mj*Vj*Wj;
      p.rho[j] += mi*Vi*Wi;
      vol1[i] += Vj*Vj*Wj;
      vol1[j] += Vi*Vi*Wi;
    }
    const double W0 = p.W.kernelValue(0.0, Hdeti);
    wsum[i] += Vi*W0;
    vol1[i] = (vol1[i] + Vi*Vi*W0)/wsum[i];
    p.rho[i] = std::max(std::max(p.cfg.rhoMin, 0.1*mi*sdet(p.H[i])),
                        std::min(p.cfg.rhoMax, (p.rho[i] + mi*Vi*W0)/(wsum[i]*vol1[i])));
  }
}

void crkMoments(Problem& p) {
  const int n = numNodes(p);
  p.m0.assign(n, 0.0); p.m1.assign(n, V3{0, 0, 0}); p.cm2.assign(n, Sym{0, 0, 0, 0, 0, 0});
  p.gradm0.assign(n, V3{0, 0, 0}); p.gradm1.assign(n, tzero());
  std::array<double, 27> z{};
  p.gradm2.assign(n, z);
  const double fij = 1.0;
  for (int i = 0; i < p.nInt; ++i) {
    const double weighti = p.vol[i];
    const V3& ri = p.pos[i];
    const Sym& Hi = p.H[i];
    const double Hdeti = sdet(Hi);
    const double wwself = weighti*p.W.kernelValue(0.0, Hdeti);
    p.m0[i] += wwself;
    taddto(p.gradm1[i], tdiag(wwself));
    for (int j : p.conn[i]) {
      if (!calcPair(i, j)) continue;
      const double weightj = p.vol[j];
      const Sym& Hj = p.H[j];
      const double Hdetj = sdet(Hj);
      const double wi = weighti, wj = weightj;
      const V3 rij = vsub(ri, p.pos[j]);
      const V3 etai = sdot(Hi, rij);
      const V3 etaj = sdot(Hj, rij);
      const auto WWi = p.W.kernelAndGradValue(mag(etai), Hdeti);
      const auto WWj = p.W.kernelAndGradValue(mag(etaj), Hdetj);
      const double Wi = 0.5*(WWi.first + WWj.first);
      const double Wj = Wi;
      const V3 gradWj = vmul(vadd(vmul(sdot(Hj, unitVector(etaj)), WWj.second),
                                  vmul(sdot(Hi, unitVector(etai)), WWi.second)), 0.5);
      const V3 gradWi = vneg(gradWj);
      const double wwi = wi*Wi, wwj = wj*Wj;
      p.m0[i] += fij*wwj;
      p.m0[j] += fij*wwi;
      for (int ii = 0; ii < 3; ++ii) {
        el(p.gradm0[i], ii) += fij*wj*el(gradWj, ii);
        el(p.gradm0[j], ii) += fij*wi*el(gradWi, ii);
      }
      for (int ii = 0; ii < 3; ++ii) {
        el(p.m1[i], ii) += fij*wwj*el(rij, ii);
        el(p.m1[j], ii) -= fij*wwi*el(rij, ii);
        for (int jj = 0; jj < 3; ++jj) {
          el(p.gradm1[i], ii, jj) += fij*wj*el(rij, ii)*el(gradWj, jj);
          el(p.gradm1[j], ii, jj) -= fij*wi*el(rij, ii)*el(gradWi, jj);
        }
        el(p.gradm1[i], ii, ii) += fij*wj*Wj;
        el(p.gradm1[j], ii, ii) += fij*wi*Wi;
      }
      for (int ii = 0; ii < 3; ++ii) {
        for (int jj = ii; jj < 3; ++jj) {
          const double thpt = el(rij, ii)*el(rij, jj);
          sel(p.cm2[i], ii, jj) += fij*wwj*thpt;
          sel(p.cm2[j], ii, jj) += fij*wwi*thpt;
        }
        for (int jj = 0; jj < 3; ++jj) {
          const double thpt = el(rij, ii)*el(rij, jj);
          for (int kk = 0; kk < 3; ++kk) {
            p.gradm2[i][9*ii + 3*jj + kk] += fij*wj*thpt*el(gradWj, kk);
            p.gradm2[j][9*ii + 3*jj + kk] += fij*wi*thpt*el(gradWi, kk);
          }
          p.gradm2[i][9*ii + 3*jj + jj] += fij*wwj*el(rij, ii);
          p.gradm2[i][9*jj + 3*ii + jj] += fij*wwj*el(rij, ii);
          p.gradm2[j][9*ii + 3*jj + jj] -= fij*wwi*el(rij, ii);
          p.gradm2[j][9*jj + 3*ii + jj] -= fij*wwi*el(rij, ii);
        }
      }
    }
  }
}

void crkCorrections(Problem& p) {
  crkResize(p);
  for (int i = 0; i < p.nInt; ++i) {
    const V3& m1i = p.m1[i];
    const Sym& m2i = p.cm2[i];
    const double Hd = sdet(p.H[i]);
    const double hdet2 = 1.0/(Hd*Hd);
    const double m2det = sdet(m2i);
    const Sym m2inv = std::abs(m2det) > 1.0e-5*hdet2 ? sinverse(m2i) : Sym{0, 0, 0, 0, 0, 0};
    const V3 m2invm1 = sdot(m2inv, m1i);
    const double Ainv = p.m0[i] - dot(m2invm1, m1i);
    double& A = p.A[i];
    A = 1.0/Ainv;
    p.B[i] = vneg(m2invm1);
    V3& gA = p.gradA[i];
    gA = vmul(p.gradm0[i], -A*A);
    T9& gB = p.gradB[i];
    gB = tzero();
    const T9& gm1 = p.gradm1[i];
    const std::array<double, 27>& gm2 = p.gradm2[i];
    for (int ii = 0; ii < 3; ++ii) {
      for (int jj = 0; jj < 3; ++jj) {
        for (int kk = 0; kk < 3; ++kk) {
          el(gA, ii) += A*A*sel(m2inv, jj, kk)*el(m1i, kk)*el(gm1, jj, ii);
          el(gA, ii) += A*A*sel(m2inv, jj, kk)*el(gm1, kk, ii)*el(m1i, jj);
          el(gB, ii, jj) -= sel(m2inv, ii, kk)*el(gm1, kk, jj);
          for (int ll = 0; ll < 3; ++ll) {
            for (int mm = 0; mm < 3; ++mm) {
              el(gA, ii) -= A*A*sel(m2inv, jj, kk)*gm2[9*kk + 3*ll + ii]*sel(m2inv, ll, mm)*el(m1i, mm)*el(m1i, jj);
              el(gB, ii, jj) += sel(m2inv, ii, kk)*gm2[9*kk + 3*ll + jj]*sel(m2inv, ll, mm)*el(m1i, mm);
            }
          }
        }
      }
    }
  }
  ghostCopy(p, p.A); ghostCopy(p, p.B); ghostCopy(p, p.gradA); ghostCopy(p, p.gradB);
}

// CRKSPHKernelAndGradient, LinearOrder, no correction limits in effect.
void crkKernel(const TableKernel& W, const V3& rij, const V3& etai, const Sym& Hi, double Hdeti,
               const V3& etaj, const Sym& Hj, double Hdetj, double Ai, const V3& Bi, const V3& gradAi,
               const T9& gradBi, double& WCRK, double& gradWSPH, V3& gradWCRK) {
  const double correctionMin = -DBL_MAX, correctionMax = DBL_MAX;
  const auto WWi = W.kernelAndGradValue(mag(etai), Hdeti);
  const auto WWj = W.kernelAndGradValue(mag(etaj), Hdetj);
  const double Wij = 0.5*(WWi.first + WWj.first);
  const V3 gradWij = vmul(vadd(vmul(sdot(Hi, unitVector(etai)), WWi.second),
                               vmul(sdot(Hj, unitVector(etaj)), WWj.second)), 0.5);
  gradWSPH = 0.5*(WWi.second + WWj.second);
  const double correction0 = Ai*(1.0 + dot(Bi, rij));
  const double correction = std::max(correctionMin, std::min(correctionMax, correction0));
  WCRK = correction*Wij;
  gradWCRK = vmul(gradWij, correction);
  if (correction0 > correctionMin && correction0 < correctionMax) {
    gradWCRK = vadd(gradWCRK, vadd(vmul(vmul(Bi, Ai), Wij), vmul(vmul(gradAi, 1.0 + dot(Bi, rij)), Wij)));
    for (int ii = 0; ii < 3; ++ii)
      for (int jj = 0; jj < 3; ++jj)
        el(gradWCRK, ii) += Ai*Wij*el(gradBi, jj, ii)*el(rij, jj);
  }
}

// CRKSPHMonaghanGingoldViscosity::Piij velocity reconstruction
// (src/ArtificialViscosity/CRKSPHMonaghanGingoldViscosity.cc:223-247), pair
// (i, j) in the reference's orientation; the limited velocities then enter
// the Monaghan-Gingold mu.
inline double limiterVL(const double x) {
  if (x > 0.0) return 2.0/(1.0 + x)*2.0*x/(1.0 + x);
  return 0.0;
}
void crkQVelocities(const Problem& p, int i, int j, const V3& etai, const V3& etaj, V3& vi1, V3& vj1) {
  const T9& DvDxi = p.qGradVel[i];
  const T9& DvDxj = p.qGradVel[j];
  const V3 xij = vmul(vsub(p.pos[i], p.pos[j]), 0.5);
  const double gradi = dot(tvdot(DvDxi, xij), xij);
  const double gradj = dot(tvdot(DvDxj, xij), xij);
  const double ri = gradi/(sgn(gradj)*std::max(1.0e-30, std::abs(gradj)));
  const double rj = gradj/(sgn(gradi)*std::max(1.0e-30, std::abs(gradi)));
  double phi = limiterVL(std::min(ri, rj));
  const double etaCrit = p.cfg.etaCritFrac/p.cfg.nPerh, etaFold = p.cfg.etaFoldFrac/p.cfg.nPerh;
  const double etaij = std::min(mag(etai), mag(etaj));
  if (etaij < etaCrit) {
    const double y = (etaij - etaCrit)/etaFold;
    phi *= std::exp(-(y*y));
  }
  vi1 = vsub(p.vel[i], tvdot(tmul(DvDxi, phi), xij));
  vj1 = vadd(p.vel[j], tvdot(tmul(DvDxj, phi), xij));
}

void crkEvaluateDerivatives(Problem& p) {
  zeroDerivs(p);
  const int n = numNodes(p);
  p.gradRho.assign(n, V3{0, 0, 0});
  const TableKernel& W = p.W;
  const double nPerh = p.cfg.nPerh;
  const bool compatible = p.cfg.compatibleEnergyEvolution != 0;
  const bool XSPH = p.cfg.XSPH != 0;
  for (int i = 0; i < p.nInt; ++i) {
    const V3& ri = p.pos[i]; const double mi = p.m[i]; const V3& vi = p.vel[i];
    const double rhoi = p.rho[i]; const double Pi = p.P[i]; const Sym& Hi = p.H[i]; const double ci = p.cs[i];
    const double Ai = p.A[i]; const V3& Bi = p.B[i]; const V3& gradAi = p.gradA[i]; const T9& gradBi = p.gradB[i];
    const double Hdeti = sdet(Hi);
    const double weighti = p.vol[i];
    for (int j : p.conn[i]) {
      if (!calcPair(i, j)) continue;
      const V3& rj = p.pos[j]; const double mj = p.m[j]; const V3& vj = p.vel[j];
      const double rhoj = p.rho[j]; const double Pj = p.P[j]; const Sym& Hj = p.H[j]; const double cj = p.cs[j];
      const double Aj = p.A[j]; const V3& Bj = p.B[j]; const V3& gradAj = p.gradA[j]; const T9& gradBj = p.gradB[j];
      const double Hdetj = sdet(Hj);
      const double weightj = p.vol[j];
      const V3 rij = vsub(ri, rj);
      const V3 etai = sdot(Hi, rij);
      const V3 etaj = sdot(Hj, rij);
      const V3 vij = vsub(vi, vj);
      double Wj, gWj, Wi, gWi;
      V3 gradWj, gradWi;
      crkKernel(W, rij, etai, Hi, Hdeti, etaj, Hj, Hdetj, Ai, Bi, gradAi, gradBi, Wj, gWj, gradWj);
      crkKernel(W, vneg(rij), vneg(etaj), Hj, Hdetj, vneg(etai), Hi, Hdeti, Aj, Bj, gradAj, gradBj, Wi, gWi, gradWi);
      const V3 deltagrad = vsub(gradWj, gradWi);
      const V3 gradWSPHi = vmul(sdot(Hi, unitVector(etai)), W.gradValue(mag(etai), Hdeti));
      const V3 gradWSPHj = vmul(sdot(Hj, unitVector(etaj)), W.gradValue(mag(etaj), Hdetj));
      {
        const double fweightij = 1.0;
        const double rij2 = mag2(rij);
        const Sym thpt = smul(selfdyad(rij), safeInvVar(rij2*rij2*rij2));
        p.wns[i] += fweightij*std::abs(gWi);
        p.wns[j] += 1.0/fweightij*std::abs(gWj);
        p.m2[i] = sadd(p.m2[i], smul(thpt, fweightij*mag2(gradWSPHi)));
        p.m2[j] = sadd(p.m2[j], smul(thpt, 1.0/fweightij*mag2(gradWSPHj)));
      }
      T9 QPi, QPj;
      if (p.cfg.qType == SPHGPU_Q_CRKSPH_MONAGHAN_GINGOLD) {
        V3 vi1, vj1;
        crkQVelocities(p, i, j, etai, etaj, vi1, vj1);
        Piij(p, etai, vi1, rhoi, ci, etaj, vj1, rhoj, cj, QPi, QPj);
      } else {
        Piij(p, etai, vi, rhoi, ci, etaj, vj, rhoj, cj, QPi, QPj);
      }
      T9 Qsum = tmul(QPi, rhoi*rhoi);
      taddto(Qsum, tmul(QPj, rhoj*rhoj));
      const V3 Qaccij = tvdot(Qsum, deltagrad);
      const double workQi = rhoj*rhoj*dot(tvdot(QPj, vij), deltagrad);
      const double workQj = rhoi*rhoi*dot(tvdot(QPi, vij), deltagrad);
      const double Qi = rhoi*rhoi*(maxAbsElement(V3{QPi.xx, QPi.yy, QPi.zz}));
      const double Qj = rhoj*rhoj*(maxAbsElement(V3{QPj.xx, QPj.yy, QPj.zz}));
      p.maxvp[i] = std::max(p.maxvp[i], 4.0*Qi);
      p.maxvp[j] = std::max(p.maxvp[j], 4.0*Qj);
      p.effvp[i] += weightj*Qi*Wj;
      p.effvp[j] += weighti*Qj*Wi;
      p.viscW[i] += 0.5*weighti*weightj/mi*workQi;
      p.viscW[j] += 0.5*weighti*weightj/mj*workQj;
      const T9 deltaDvDxi = tmul(dyad(vij, gradWj), -weightj);
      const T9 deltaDvDxj = tmul(dyad(vij, gradWi), weighti);
      taddto(p.DvDx[i], deltaDvDxi);
      taddto(p.DvDx[j], deltaDvDxj);
      taddto(p.localDvDx[i], deltaDvDxi);
      taddto(p.localDvDx[j], deltaDvDxj);
      p.gradRho[i] = vadd(p.gradRho[i], vmul(gradWj, weightj*(rhoj - rhoi)));
      p.gradRho[j] = vadd(p.gradRho[j], vmul(gradWi, weighti*(rhoi - rhoj)));
      const V3 forceij = vmul(vadd(vmul(deltagrad, Pi + Pj), Qaccij), 0.5*weighti*weightj);
      const V3 forceji = vmul(vadd(vmul(deltagrad, Pi + Pj), Qaccij), 0.5*weighti*weightj);
      p.DvDt[i] = vsub(p.DvDt[i], vdiv(forceij, mi));
      p.DvDt[j] = vadd(p.DvDt[j], vdiv(forceji, mj));
      if (compatible) {
        p.pairAcc[i].push_back(vdiv(vneg(forceij), mi));
        p.pairAcc[j].push_back(vdiv(forceji, mj));
      }
      p.DepsDt[i] += 0.5*weighti*weightj*(Pj*dot(vij, deltagrad) + workQi)/mi;
      p.DepsDt[j] += 0.5*weighti*weightj*(Pi*dot(vij, deltagrad) + workQj)/mj;
      if (XSPH) {
        p.XSPHdv[i] = vsub(p.XSPHdv[i], vmul(vij, weightj*Wj));
        p.XSPHdv[j] = vadd(p.XSPHdv[j], vmul(vij, weighti*Wi));
      }
    }
    p.DrhoDt[i] = -rhoi*ttrace(p.DvDx[i]);
    p.wns[i] = CubeRootHalley2(std::max(0.0, p.wns[i]/Hdeti));
    p.m2[i] = sdiv(p.m2[i], Hdeti*Hdeti);
    p.DxDt[i] = XSPH ? vadd(vi, p.XSPHdv[i]) : vi;
    p.DHDt[i] = smul(sdiv(sneg(Hi), 3), ttrace(p.DvDx[i]));
    const double zerothMoment = p.wns[i];
    double cur;
    if (fuzzyEqual(zerothMoment, 0.0)) cur = 0.5*nPerh;
    else cur = W.equivalentNodesPerSmoothingScale(zerothMoment);
    const double s = std::min(4.0, std::max(0.25, nPerh/(cur + 1.0e-30)));
    double a;
    if (s < 1.0) a = 0.4*(1.0 + s*s);
    else a = 0.4*(1.0 + 1.0/(s*s*s));
    const double hi0 = 1.0/Hi.xx;
    const double hi1 = std::min(p.cfg.hmax, std::max(p.cfg.hmin, hi0*(1.0 - a + a*s)));
    const double inv = 1.0/hi1;
    p.Hideal[i] = Sym{1.0*inv, 0.0*inv, 0.0*inv, 1.0*inv, 0.0*inv, 1.0*inv};
  }
}

// ContinuityVolumePolicy (fires after the mass density and H updates).
// CRKMassOverDensity volume: the reference forms mass/massDensity as a
// FieldList quotient, which multiplies by safeInvVar(rho, 1e-60)
// (src/Field/FieldInline.hh:614-623, src/Utilities/safeInv.hh:24-27), not a
// plain division.
double massOverDensity(double m, double rho) {
  const double s = rho > 0.0 ? 1.0 : (rho < 0.0 ? -1.0 : 0.0);
  return m*(s/std::max(1.0e-60, std::fabs(rho)));
}

void crkVolumeUpdate(Problem& p, double multiplier) {
  for (int i = 0; i < p.nInt; ++i) {
    const double volMin = 0.5*p.m[i]*safeInvVar(p.rho[i]);
    const double volMax = 4.0*M_PI/(3.0*sdet(p.H[i]));
    const double dVdt = -p.m[i]*safeInvVar(p.rho[i]*p.rho[i])*p.DrhoDt[i];
    p.vol[i] = std::max(volMin, std::min(volMax, p.vol[i] + multiplier*dVdt));
  }
}

void crkInitialize(Problem& p) {
  crkMoments(p);
  crkCorrections(p);
  // CRKSPHMonaghanGingoldViscosity::initialize
  // (src/ArtificialViscosity/CRKSPHMonaghanGingoldViscosity.cc:119-150): cache
  // the last velocity gradient, ghosts by the boundary copies.
  if (p.cfg.qType == SPHGPU_Q_CRKSPH_MONAGHAN_GINGOLD) {
    p.qGradVel.assign(numNodes(p), tzero());
    for (int i = 0; i < p.nInt && i < int(p.DvDx.size()); ++i) p.qGradVel[i] = p.DvDx[i];
    ghostCopy(p, p.qGradVel);
  }
}



bool crkStepRK2(Problem& p, double& dtOut) {
  const double t = p.time;
  preStepInitialize(p);
  crkResize(p);
  ghostCopy(p, p.vol);
  const double dt = selectDt(p);
  const double hdt = 0.5*dt;
  const std::vector<V3> pos0 = p.pos, vel0 = p.vel;
  const std::vector<double> rho0 = p.rho, eps0 = p.eps, P0 = p.P, cs0 = p.cs, vol0 = p.vol;
  const std::vector<Sym> H0 = p.H;
  if (!stateUpdate(p, hdt, true)) return false;
  crkVolumeUpdate(p, hdt);
  p.time = t + hdt;
  applyGhostBoundaries(p);
  ghostCopy(p, p.vol);
  crkInitialize(p);
  crkEvaluateDerivatives(p);
  finalizeDerivatives(p);
  p.pos = pos0; p.vel = vel0; p.rho = rho0; p.eps = eps0; p.P = P0; p.cs = cs0; p.H = H0; p.vol = vol0;
  if (!stateUpdate(p, dt, false)) return false;
  crkVolumeUpdate(p, dt);
  p.time = t + dt;
  applyGhostBoundaries(p);
  ghostCopy(p, p.vol);
  // CRKSPHHydroBase::finalize (src/CRKSPH/CRKSPHHydroBase.cc:1213-1216): the
  // volume of the configured type, then the summed density.
  if (p.cfg.crkVolumeType == SPHGPU_CRK_SUMVOLUME) crkSumVolume(p);
  else for (int i = 0; i < numNodes(p); ++i) p.vol[i] = massOverDensity(p.m[i], p.rho[i]);
  if (p.cfg.densityUpdate == SPHGPU_DENSITY_RIGOROUS_SUM) crkSumDensity(p);
  enforceBoundaries(p);
  p.cycle += 1;
  p.lastDt = dt;
  dtOut = dt;
  return true;
}

}  // namespace

// ============================================================== C API
// iterateIdealH (src/Utilities/iterateIdealH.cc:26-349) with the drivers'
// arguments (SpheralController.iterateIdealH: nPerhForIteration = 0,
// sphericalStart = false, fixDeterminant = false) and SPHSmoothingScale
// (src/NodeList/SPHSmoothingScale.cc:102-225).  One NodeList, so every
// neighbor weight fweightij is 1 and the second moment (unused by the SPH
// smoothing scale) is not formed.  Each iteration rebuilds the ghosts and
// the ConnectivityMap from the current H; nodes whose last change was within
// the tolerance keep their H.  The change of H is measured as the reference
// does: phi = eig((H1^1/2 Hi^-1 H1^1/2).Symmetric()), with H1 = c I from the
// ideal smoothing scale, whose square root comes from a diagonal eigen
// decomposition (eigenvalue (c*(1/c))*c, identity eigenvectors).
int iterateIdealH(Problem& p, int maxIterations, double tolerance, double* maxDeltaHOut) {
  const int nInt = p.nInt;
  std::vector<double> deltaH(nInt, 2.0*tolerance);
  const double nPerh = p.cfg.nPerh;
  int itr = 0;
  double maxDeltaH = 2.0*tolerance;
  while (itr < maxIterations && maxDeltaH > tolerance) {
    ++itr;
    maxDeltaH = 0.0;
    preStepInitialize(p);
    std::vector<Sym> H1(p.H.begin(), p.H.begin() + nInt);
    for (int i = 0; i < nInt; ++i) {
      if (deltaH[i] <= tolerance) continue;
      const V3& posi = p.pos[i];
      const Sym& Hi = p.H[i];
      double zerothMoment = 0.0;
      for (int j : p.conn[i]) {
        const V3 xij = vsub(posi, p.pos[j]);
        const double etai = mag(sdot(Hi, xij));
        const double Wi = std::abs(p.W.gradValue(etai, 1.0));
        zerothMoment += Wi;
      }
      zerothMoment = CubeRootHalley2(zerothMoment);        // Dim<3>::rootnu
      double currentNodesPerSmoothingScale;
      if (fuzzyEqual(zerothMoment, 0.0)) currentNodesPerSmoothingScale = 0.5*nPerh;
      else currentNodesPerSmoothingScale = p.W.equivalentNodesPerSmoothingScale(zerothMoment);
      const double s = std::min(4.0, std::max(0.25, nPerh/(currentNodesPerSmoothingScale + 1.0e-30)));
      double a;
      if (s < 1.0) a = 0.4*(1.0 + s*s);
      else a = 0.4*(1.0 + 1.0/(s*s*s));
      const double hi0 = 1.0/Hi.xx;
      const double hi1 = std::min(p.cfg.hmax, std::max(p.cfg.hmin, hi0*(1.0 - a + a*s)));
      const double inv = 1.0/hi1;
      H1[i] = Sym{1.0*inv, 0.0*inv, 0.0*inv, 1.0*inv, 0.0*inv, 1.0*inv};
      // H1.sqrt(): eigen decomposition of the scaled diagonal tensor
      const double fscale = std::max(10.0*2.220446049250313e-16, smaxAbsElement(H1[i]));
      const double lam = (inv*(1.0/fscale))*fscale;
      const double r = std::sqrt(lam);
      const Sym Hinv = sinverse(Hi);
      const Sym S{r*(r*Hinv.xx), r*(r*Hinv.xy), r*(r*Hinv.xz), r*(r*Hinv.yy), r*(r*Hinv.yz), r*(r*Hinv.zz)};
      const V3 phi = eigenValues(S);
      const double deltaHi = std::max(std::abs(minElement(phi) - 1.0), std::abs(maxElement(phi) - 1.0));
      deltaH[i] = deltaHi;
      maxDeltaH = std::max(maxDeltaH, deltaHi);
    }
    for (int i = 0; i < nInt; ++i) p.H[i] = H1[i];
  }
  p.haveConn = false;
  if (maxDeltaHOut) *maxDeltaHOut = maxDeltaH;
  return itr;
}

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

void* orc_create(const sphgpu_config* cfg, int n, const double* pos, const double* vel,
                 const double* mass, const double* rho, const double* eps, const double* H) {
  Problem* p = new Problem();
  p->cfg = *cfg;
  p->W = TableKernel(cfg->kernel, cfg->num_points);
  p->nInt = n;
  resizeAll(*p, n);
  for (int i = 0; i < n; ++i) {
    p->pos[i] = V3{pos[3*i], pos[3*i + 1], pos[3*i + 2]};
    p->vel[i] = V3{vel[3*i], vel[3*i + 1], vel[3*i + 2]};
    p->m[i] = mass[i]; p->rho[i] = rho[i]; p->eps[i] = eps[i];
    p->H[i] = Sym{H[6*i], H[6*i + 1], H[6*i + 2], H[6*i + 3], H[6*i + 4], H[6*i + 5]};
    p->omega[i] = 1.0;
  }
  updateEOS(*p, 0, n);
  p->lastDt = cfg->lastDt;
  makeBoundaries(*p);
  zeroDerivs(*p);
  return p;
}

void orc_destroy(void* h) { delete static_cast<Problem*>(h); }

// Integrator::setGhostNodes + ConnectivityMap + applyGhostBoundaries.
int orc_build_neighbors(void* h) {
  Problem& p = *static_cast<Problem*>(h);
  preStepInitialize(p);
  if (p.cfg.hydro == SPHGPU_HYDRO_CRKSPH) {
    // CRKSPHHydroBase::initializeProblemStartup volumes (first call) and the
    // ghost copy of the evolved volume afterwards.
    crkResize(p);
    if (!p.crkVolumeReady) {
      if (p.cfg.crkVolumeType == SPHGPU_CRK_SUMVOLUME) crkSumVolume(p);
      else for (int i = 0; i < numNodes(p); ++i) p.vol[i] = massOverDensity(p.m[i], p.rho[i]);
      p.crkVolumeReady = true;
    }
    ghostCopy(p, p.vol);
  }
  return 0;
}

int orc_iterate_ideal_h(void* h, int maxIterations, double tolerance, double* maxDeltaH) {
  Problem& p = *static_cast<Problem*>(h);
  return iterateIdealH(p, maxIterations, tolerance, maxDeltaH);
}

int orc_num_ghosts(void* h) { Problem& p = *static_cast<Problem*>(h); return numNodes(p) - p.nInt; }
int64_t orc_num_entries(void* h) {
  Problem& p = *static_cast<Problem*>(h);
  int64_t e = 0;
  for (auto& r : p.conn) e += int64_t(r.size());
  return e;
}
int64_t orc_num_pairs(void* h) {
  Problem& p = *static_cast<Problem*>(h);
  int64_t e = 0;
  for (int i = 0; i < p.nInt; ++i) for (int j : p.conn[i]) e += (j > i);
  return e;
}

int orc_get_connectivity(void* h, int64_t* offsets, int32_t* nbrs, int32_t* ghostRoot) {
  Problem& p = *static_cast<Problem*>(h);
  int64_t o = 0;
  for (int i = 0; i < p.nInt; ++i) {
    if (offsets) offsets[i] = o;
    for (int j : p.conn[i]) { if (nbrs) nbrs[o] = j; ++o; }
  }
  if (offsets) offsets[p.nInt] = o;
  if (ghostRoot) {
    std::vector<int> root(numNodes(p));
    for (int i = 0; i < p.nInt; ++i) root[i] = i;
    for (size_t b = 0; b < p.bcs.size(); ++b)
      for (size_t k = 0; k < p.control[b].size(); ++k) root[p.ghosts[b][k]] = root[p.control[b][k]];
    for (int g = p.nInt; g < numNodes(p); ++g) ghostRoot[g - p.nInt] = root[g];
  }
  return 0;
}

int orc_get_ghost_positions(void* h, double* out) {
  Problem& p = *static_cast<Problem*>(h);
  for (int g = p.nInt; g < numNodes(p); ++g) {
    out[3*(g - p.nInt)] = p.pos[g].x; out[3*(g - p.nInt) + 1] = p.pos[g].y; out[3*(g - p.nInt) + 2] = p.pos[g].z;
  }
  return 0;
}

int orc_initialize(void* h) {
  Problem& p = *static_cast<Problem*>(h);
  if (p.cfg.hydro == SPHGPU_HYDRO_CRKSPH) crkInitialize(p);
  else initializeDerivatives(p);
  return 0;
}
int orc_evaluate_derivatives(void* h) {
  Problem& p = *static_cast<Problem*>(h);
  if (p.cfg.hydro == SPHGPU_HYDRO_CRKSPH) crkEvaluateDerivatives(p);
  else evaluateDerivatives(p);
  finalizeDerivatives(p);
  return 0;
}
int orc_finalize(void* h) {
  Problem& p = *static_cast<Problem*>(h);
  if (p.cfg.hydro == SPHGPU_HYDRO_CRKSPH) {
    if (p.cfg.crkVolumeType == SPHGPU_CRK_SUMVOLUME) crkSumVolume(p);
    else for (int i = 0; i < numNodes(p); ++i) p.vol[i] = massOverDensity(p.m[i], p.rho[i]);
    if (p.cfg.densityUpdate == SPHGPU_DENSITY_RIGOROUS_SUM) crkSumDensity(p);
  } else {
    finalizeStep(p);
  }
  return 0;
}
double orc_dt(void* h) { return hydroDt(*static_cast<Problem*>(h)); }

int orc_step_rk2(void* h, int nsteps, double* time, double* lastDt) {
  Problem& p = *static_cast<Problem*>(h);
  double dt = 0.0;
  for (int s = 0; s < nsteps; ++s) {
    const bool ok = p.cfg.hydro == SPHGPU_HYDRO_CRKSPH ? crkStepRK2(p, dt) : stepRK2(p, dt);
    if (!ok) return -6;
  }
  if (time) *time = p.time;
  if (lastDt) *lastDt = dt;
  return 0;
}

// Field access by the reference's key (internal nodes only).
int orc_get_field(void* h, const char* key, double* out) {
  Problem& p = *static_cast<Problem*>(h);
  const std::string k(key);
  const int n = p.nInt;
  auto S = [&](const std::vector<double>& f) { for (int i = 0; i < n; ++i) out[i] = f[i]; return 0; };
  auto V = [&](const std::vector<V3>& f) {
    for (int i = 0; i < n; ++i) { out[3*i] = f[i].x; out[3*i + 1] = f[i].y; out[3*i + 2] = f[i].z; } return 0; };
  auto Y = [&](const std::vector<Sym>& f) {
    for (int i = 0; i < n; ++i) { const Sym& s = f[i]; double* o = out + 6*i;
      o[0] = s.xx; o[1] = s.xy; o[2] = s.xz; o[3] = s.yy; o[4] = s.yz; o[5] = s.zz; } return 0; };
  auto T = [&](const std::vector<T9>& f) {
    for (int i = 0; i < n; ++i) { const T9& t = f[i]; double* o = out + 9*i;
      o[0] = t.xx; o[1] = t.xy; o[2] = t.xz; o[3] = t.yx; o[4] = t.yy; o[5] = t.yz; o[6] = t.zx; o[7] = t.zy; o[8] = t.zz; }
    return 0; };
  if (k == "position") return V(p.pos);
  if (k == "velocity") return V(p.vel);
  if (k == "mass") return S(p.m);
  if (k == "mass density") return S(p.rho);
  if (k == "specific thermal energy") return S(p.eps);
  if (k == "H") return Y(p.H);
  if (k == "pressure") return S(p.P);
  if (k == "sound speed") return S(p.cs);
  if (k == "grad h corrections") return S(p.omega);
  if (k == "new mass density") return S(p.rhoSum);
  if (k == "normalization") return S(p.norm);
  if (k == "delta position") return V(p.DxDt);
  if (k == "delta mass density") return S(p.DrhoDt);
  if (k == "delta velocity hydro") return V(p.DvDt);
  if (k == "delta specific thermal energy") return S(p.DepsDt);
  if (k == "velocity gradient") return T(p.DvDx);
  if (k == "internal velocity gradient") return T(p.localDvDx);
  if (k == "M SPH gradient correction") return T(p.M);
  if (k == "local M SPH gradient correction") return T(p.localM);
  if (k == "delta H") return Y(p.DHDt);
  if (k == "new H") return Y(p.Hideal);
  if (k == "max viscous pressure") return S(p.maxvp);
  if (k == "effective viscous pressure") return S(p.effvp);
  if (k == "viscous work rate") return S(p.viscW);
  if (k == "XSPH weight sum") return S(p.XSPHw);
  if (k == "XSPH delta vi") return V(p.XSPHdv);
  if (k == "weighted neighbor sum") return S(p.wns);
  if (k == "mass second moment") return Y(p.m2);
  if (k == "node volume") return S(p.vol);
  if (k == "A CRKSPH correction") return S(p.A);
  if (k == "B CRKSPH correction") return V(p.B);
  if (k == "grad A CRKSPH correction") return V(p.gradA);
  if (k == "grad B CRKSPH correction") return T(p.gradB);
  if (k == "m0 CRKSPH moment") return S(p.m0);
  if (k == "m1 CRKSPH moment") return V(p.m1);
  if (k == "m2 CRKSPH moment") return Y(p.cm2);
  if (k == "grad m0 CRKSPH moment") return V(p.gradm0);
  if (k == "grad m1 CRKSPH moment") return T(p.gradm1);
  if (k == "mass density gradient") return V(p.gradRho);
  if (k == "grad m2 CRKSPH moment") {
    for (int i = 0; i < n; ++i) for (int c = 0; c < 27; ++c) out[27*i + c] = p.gradm2[i][c];
    return 0;
  }
  g_err = "unknown field key " + k;
  return -1;
}

// CRK reproducing conditions at each internal node i (after orc_initialize):
// out[4i] = sum_j V_j W^R_ij (self included, should be 1),
// out[4i+1..3] = sum_j V_j W^R_ij (r_j - r_i) (should vanish), with
// W^R_ij = A_i (1 + B_i . r_ij) W_ij and W_ij the symmetrized kernel.
int orc_crk_reproduction(void* h, double* out) {
  Problem& p = *static_cast<Problem*>(h);
  for (int i = 0; i < p.nInt; ++i) {
    const double Hdeti = sdet(p.H[i]);
    double s0 = p.vol[i]*p.A[i]*p.W.kernelValue(0.0, Hdeti);
    V3 s1{0, 0, 0};
    for (int j : p.conn[i]) {
      const V3 rij = vsub(p.pos[i], p.pos[j]);
      const double Wij = 0.5*(p.W.kernelValue(mag(sdot(p.H[i], rij)), Hdeti) +
                              p.W.kernelValue(mag(sdot(p.H[j], rij)), sdet(p.H[j])));
      const double WR = p.A[i]*(1.0 + dot(p.B[i], rij))*Wij;
      s0 += p.vol[j]*WR;
      s1 = vadd(s1, vmul(vneg(rij), p.vol[j]*WR));
    }
    out[4*i] = s0; out[4*i + 1] = s1.x; out[4*i + 2] = s1.y; out[4*i + 3] = s1.z;
  }
  return 0;
}

// Pair-wise accelerations per node, flattened in the reference's push order
// (node i: j-side pushes from lower owners, then its own pushes).
int orc_get_pair_accelerations(void* h, double* out) {
  Problem& p = *static_cast<Problem*>(h);
  int64_t o = 0;
  for (int i = 0; i < p.nInt; ++i)
    for (const V3& a : p.pairAcc[i]) { out[3*o] = a.x; out[3*o + 1] = a.y; out[3*o + 2] = a.z; ++o; }
  return 0;
}

int orc_conservation(void* h, double* out) {
  Problem& p = *static_cast<Problem*>(h);
  double M = 0, px = 0, py = 0, pz = 0, KE = 0, TE = 0;
  for (int i = 0; i < p.nInt; ++i) {
    M += p.m[i];
    px += p.m[i]*p.vel[i].x; py += p.m[i]*p.vel[i].y; pz += p.m[i]*p.vel[i].z;
    KE += 0.5*p.m[i]*mag2(p.vel[i]);
    TE += p.m[i]*p.eps[i];
  }
  out[0] = M; out[1] = px; out[2] = py; out[3] = pz; out[4] = KE; out[5] = TE; out[6] = KE + TE; out[7] = 0.0;
  return 0;
}

// ---- TableKernel access (for the kernel-table known-answer tests)
void* orc_table_create(int kernelType, int numPoints) { return new TableKernel(kernelType, numPoints); }
void orc_table_destroy(void* t) { delete static_cast<TableKernel*>(t); }
int orc_table_coeffs(void* t, double* out) {
  // out: 9 arrays of numPoints (aK,bK,cK,aG,bG,cG,aG2,bG2,cG2) then nperh, wsum
  TableKernel& W = *static_cast<TableKernel*>(t);
  const std::vector<double>* v[11] = {&W.aK, &W.bK, &W.cK, &W.aG, &W.bG, &W.cG, &W.aG2, &W.bG2, &W.cG2, &W.nperh, &W.wsum};
  for (int k = 0; k < 11; ++k) std::memcpy(out + size_t(k)*W.n, v[k]->data(), sizeof(double)*W.n);
  return 0;
}
int orc_table_eval(void* t, int n, const double* eta, double Hdet, double* Wout, double* gWout, double* nperhOut) {
  TableKernel& W = *static_cast<TableKernel*>(t);
  for (int i = 0; i < n; ++i) {
    const auto r = W.kernelAndGradValue(eta[i], Hdet);
    if (Wout) Wout[i] = r.first;
    if (gWout) gWout[i] = r.second;
    if (nperhOut) nperhOut[i] = W.equivalentNodesPerSmoothingScale(eta[i]);
  }
  return 0;
}
double orc_base_kernel(int kernelType, int which, double eta) {
  BaseKernel k(kernelType);
  return which == 0 ? k.kernelValue(eta, 1.0) : (which == 1 ? k.gradValue(eta, 1.0) : k.grad2Value(eta, 1.0));
}

// Geometry spot checks (for pinning against the reference's own headers).
int orc_geometry(int n, const double* H6, const double* r3, double* out) {
  // per sample: eigenValues(3), det(1), inverse(6), H*r (3), unitVector(r) (3)
  for (int i = 0; i < n; ++i) {
    const Sym s{H6[6*i], H6[6*i + 1], H6[6*i + 2], H6[6*i + 3], H6[6*i + 4], H6[6*i + 5]};
    const V3 r{r3[3*i], r3[3*i + 1], r3[3*i + 2]};
    double* o = out + 16*i;
    const V3 ev = eigenValues(s);
    o[0] = ev.x; o[1] = ev.y; o[2] = ev.z;
    o[3] = sdet(s);
    const Sym inv = sinverse(s);
    o[4] = inv.xx; o[5] = inv.xy; o[6] = inv.xz; o[7] = inv.yy; o[8] = inv.yz; o[9] = inv.zz;
    const V3 hr = sdot(s, r);
    o[10] = hr.x; o[11] = hr.y; o[12] = hr.z;
    const V3 u = unitVector(r);
    o[13] = u.x; o[14] = u.y; o[15] = u.z;
  }
  return 0;
}

// mapPositionThroughPlanes for the periodic planes of a box (ghost images).
int orc_map_positions(int n, const double* pos, const double* xmin, const double* xmax, int axis, int which, double* out) {
  V3 n0{0, 0, 0}, n1{0, 0, 0};
  (&n0.x)[axis] = 1.0; (&n1.x)[axis] = -1.0;
  const Plane plane1(V3{xmin[0], xmin[1], xmin[2]}, n0), plane2(V3{xmax[0], xmax[1], xmax[2]}, n1);
  const Plane& enter = which == 0 ? plane1 : plane2;
  const Plane& exit = which == 0 ? plane2 : plane1;
  for (int i = 0; i < n; ++i) {
    const V3 g = mapPositionThroughPlanes(V3{pos[3*i], pos[3*i + 1], pos[3*i + 2]}, exit, enter);
    out[3*i] = g.x; out[3*i + 1] = g.y; out[3*i + 2] = g.z;
  }
  return 0;
}

}  // extern "C"
