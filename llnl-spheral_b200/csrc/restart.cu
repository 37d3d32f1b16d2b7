// Restart files in the reference's own layout.
//
// The reference writes a restart file by RestartRegistrar::dumpState
// (src/DataOutput/RestartRegistrar.cc:155-171): every registered object, in
// priority then registration order, dumps its state under its unique label
// (RestartRegistrar::uniqueLabels, :113-131).  With FlatFileIO
// (src/FileIO/FlatFileIO.cc) in its ascii form a value is one line
// "path value" (writeGenericType, :917-925), written with precision 20; a
// Field is "path n v0 v1 ... " (operator<<, src/Field/FieldInline.hh:
// 1918-1933); vectors and tensors are "( a b c )" (src/Geometry/
// GeomVectorInline.hh operator<<, GeomSymmetricTensorInline_default.hh:
// 2270-2281); a FieldList is path/NodeListNames "name|" plus a terminating
// NUL, then path/Field0 (src/FileIO/FileIOInline.hh:10-48); a plane is
// path/point and path/normal (src/FileIO/FileIO.cc:120-123).  A reader finds
// a path as the first line that starts with it (FlatFileIO::findPathName,
// :1019-1050) and reads the value after it with operator>>.
//
// A problem of this library corresponds to one FluidNodeList with its
// artificial viscosity, SPHHydroBase or CRKSPHHydroBase, one PeriodicBoundary
// per periodic axis (which registers itself and its two PlanarBoundary
// planes) and CheapSynchronousRK2, registered in that order; its file
// carries their dumpState keys:
//   NodeList::dumpState + FluidNodeList::dumpState (src/NodeList/NodeList.cc:
//     606-621, FluidNodeList.cc:180-189)
//   ArtificialViscosity::dumpState (src/ArtificialViscosity/
//     ArtificialViscosity.cc:173-179)
//   SPHHydroBase::dumpState (src/SPH/SPHHydroBase.cc:1286-1318) or
//     CRKSPHHydroBase::dumpState (src/CRKSPH/CRKSPHHydroBase.cc:1455-1485)
//   PlanarBoundary::dumpState (src/Boundary/PlanarBoundary.cc:297-301)
//   Integrator::dumpState (src/Integrator/Integrator.cc:798-806)
// The NodeList's "work" field (per-node wall-clock cost) is written as 0.
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "problem.cuh"

namespace sphgpu {
namespace {

// ---- labels

const char* q_label(const sphgpu_config& c) {
  return c.qType == SPHGPU_Q_CRKSPH_MONAGHAN_GINGOLD ? "CRKSPHMonaghanGingoldViscosity" : "MonaghanGingoldViscosity";
}
const char* hydro_label(const sphgpu_config& c) {
  return c.hydro == SPHGPU_HYDRO_CRKSPH ? "CRKSPHHydroBase" : "SPHHydroBase";
}

// The registered objects' unique labels, in dump order.
std::vector<std::string> restart_labels(const sphgpu_config& c) {
  std::vector<std::string> raw = {"FluidNodeList", q_label(c), hydro_label(c)};
  for (int a = 0; a < 3; ++a) {
    if (!c.periodic[a]) continue;
    raw.push_back("PeriodicBoundary");
    raw.push_back("PlanarBoundary");
    raw.push_back("PlanarBoundary");
  }
  raw.push_back("CheapSynchronousRK2");
  std::vector<std::string> out;
  unsigned counter = 0;
  for (std::string l : raw) {
    bool seen = false;
    for (const std::string& o : out) seen = seen || o == l;
    if (seen) l += "_" + std::to_string(counter++);
    out.push_back(l);
  }
  return out;
}

// ---- host copies of the device state

struct HostState {
  int64_t n = 0;
  std::vector<double> S, S0, D, K, Kheld;
  double s(int f, int64_t i) const { return S[f*n + i]; }
  double s0(int f, int64_t i) const { return S0[f*n + i]; }
  double d(int f, int64_t i) const { return D[f*n + i]; }
  double k(int f, int64_t i) const { return K[f*n + i]; }
};

int download_state(Problem& p, HostState& h) {
  h.n = p.n;
  h.S.resize((size_t)NSTATE*p.n);
  h.S0.resize((size_t)NSTATE*p.n);
  h.D.resize((size_t)NDERIV*p.n);
  SPH_CHECK(cudaStreamSynchronize(p.stream));
  SPH_CHECK(cudaMemcpy(h.S.data(), p.S, sizeof(double)*h.S.size(), cudaMemcpyDeviceToHost));
  SPH_CHECK(cudaMemcpy(h.S0.data(), p.S0, sizeof(double)*h.S0.size(), cudaMemcpyDeviceToHost));
  SPH_CHECK(cudaMemcpy(h.D.data(), p.D, sizeof(double)*h.D.size(), cudaMemcpyDeviceToHost));
  if (p.cfg.hydro == SPHGPU_HYDRO_CRKSPH) {
    h.K.assign((size_t)NCRK*p.n, 0.0);
    if (p.K) SPH_CHECK(cudaMemcpy(h.K.data(), p.K, sizeof(double)*h.K.size(), cudaMemcpyDeviceToHost));
    h.Kheld.assign((size_t)K_M0*p.n, 0.0);
    if (p.Kheld) SPH_CHECK(cudaMemcpy(h.Kheld.data(), p.Kheld, sizeof(double)*h.Kheld.size(), cudaMemcpyDeviceToHost));
  }
  return SPHGPU_OK;
}

// ---- writer

enum Kind { SCALAR, VECTOR, SYMTENSOR, TENSOR, INTEGER };
int comps_of(Kind k) { return k == VECTOR ? 3 : k == SYMTENSOR ? 6 : k == TENSOR ? 9 : 1; }

class FlatWriter {
 public:
  explicit FlatWriter(FILE* f) : f_(f) {}
  bool ok() const { return ok_; }
  void put(const char* s, size_t k) {
    if (ok_ && k && std::fwrite(s, 1, k, f_) != k) ok_ = false;
  }
  void put(const std::string& s) { put(s.data(), s.size()); }
  void put(char c) { put(&c, 1); }
  // an ostream at precision 20 in its default float format prints %.20g
  void real(double v) {
    char b[48];
    const int k = std::snprintf(b, sizeof(b), "%.20g", v);
    put(b, (size_t)k);
  }
  void integer(long long v) {
    char b[32];
    const int k = std::snprintf(b, sizeof(b), "%lld", v);
    put(b, (size_t)k);
  }
  void vec(const double* c, int comps) {
    put("( ", 2);
    for (int k = 0; k < comps; ++k) { real(c[k]); put(' '); }
    put(')');
  }
  // writeGenericType of a double, an int, a string, a Vector
  void value(const std::string& path, double v) { put(path); put(' '); real(v); put('\n'); }
  void value(const std::string& path, long long v) { put(path); put(' '); integer(v); put('\n'); }
  void value(const std::string& path, const std::string& s) { put(path); put(' '); put(s); put('\n'); }
  void value(const std::string& path, const double* c, int comps) { put(path); put(' '); vec(c, comps); put('\n'); }
  // a Field of n values; get(i, c) gives component c of node i
  template <class Get>
  void field(const std::string& path, int64_t n, Kind kind, Get get) {
    put(path); put(' '); integer(n); put(' ');
    const int comps = comps_of(kind);
    double c[9];
    for (int64_t i = 0; i < n; ++i) {
      if (kind == INTEGER) { integer((long long)get(i, 0)); put(' '); continue; }
      for (int k = 0; k < comps; ++k) c[k] = get(i, k);
      if (kind == SCALAR) real(c[0]); else vec(c, comps);
      put(' ');
    }
    put('\n');
  }
  // a FieldList of one Field (the NodeList's)
  template <class Get>
  void fieldList(const std::string& path, const std::string& nodeList, int64_t n, Kind kind, Get get) {
    put(path + "/NodeListNames "); put(nodeList); put('|'); put('\0'); put('\n');
    field(path + "/Field0", n, kind, get);
  }
  void emptyFieldList(const std::string& path) { put(path + "/NodeListNames \n"); }

 private:
  FILE* f_;
  bool ok_ = true;
};

// SymTensor components in the reference's storage order (xx, xy, xz, yy, yz,
// zz) are the library's; Tensors are row-major in both.
int write_restart(Problem& p, const HostState& h, FILE* f, const std::string& name) {
  const sphgpu_config& c = p.cfg;
  const int64_t n = p.n;
  const bool crk = c.hydro == SPHGPU_HYDRO_CRKSPH;
  const std::vector<std::string> labels = restart_labels(c);
  FlatWriter w(f);
  auto S = [&](int f0) { return [&h, f0](int64_t i, int k) { return h.s(f0 + k, i); }; };
  auto Dv = [&](int f0) { return [&h, f0](int64_t i, int k) { return h.d(f0 + k, i); }; };
  auto Kv = [&](int f0) { return [&h, f0](int64_t i, int k) { return h.k(f0 + k, i); }; };
  // the corrections as the reference's State holds them between steps
  auto Kh = [&](int f0) { return [&h, f0](int64_t i, int k) { return h.Kheld[(f0 + k)*h.n + i]; }; };
  auto constant = [](double v) { return [v](int64_t, int) { return v; }; };

  // FluidNodeList
  const std::string nl = labels[0];
  w.value(nl + "/name", name);
  w.value(nl + "/numNodes", (long long)n);
  w.field(nl + "/mass", n, SCALAR, S(S_M));
  w.field(nl + "/positions", n, VECTOR, S(S_X));
  w.field(nl + "/velocity", n, VECTOR, S(S_VX));
  w.field(nl + "/H", n, SYMTENSOR, S(S_H));
  w.field(nl + "/work", n, SCALAR, constant(0.0));
  w.field(nl + "/massDensity", n, SCALAR, S(S_RHO));
  w.field(nl + "/specificThermalEnergy", n, SCALAR, S(S_EPS));

  // the artificial viscosity: constant multipliers, no shear correction
  const std::string q = labels[1];
  w.fieldList(q + "/ClMultiplier", name, n, SCALAR, constant(1.0));
  w.fieldList(q + "/CqMultiplier", name, n, SCALAR, constant(1.0));
  w.fieldList(q + "/shearCorrection", name, n, SCALAR, constant(1.0));

  // the hydro
  const std::string hy = labels[2];
  auto eps0 = [&h, &c](int64_t i, int) { return c.compatibleEnergyEvolution ? h.s0(S_EPS, i) : 0.0; };
  auto entropy = [&h](int64_t i, int) { return h.s0(S0_ENTROPY, i); };
  w.fieldList(hy + "/timeStepMask", name, n, INTEGER, constant(1.0));
  w.fieldList(hy + "/pressure", name, n, SCALAR, S(S_P));
  w.fieldList(hy + "/soundSpeed", name, n, SCALAR, S(S_CS));
  if (!crk) {
    w.emptyFieldList(hy + "/volume");
    w.fieldList(hy + "/specificThermalEnergy0", name, n, SCALAR, eps0);
    w.fieldList(hy + "/entropy", name, n, SCALAR, entropy);
    w.fieldList(hy + "/Hideal", name, n, SYMTENSOR, Dv(D_HIDEAL));
    w.fieldList(hy + "/massDensitySum", name, n, SCALAR, Dv(D_RHOSUM));
    w.fieldList(hy + "/normalization", name, n, SCALAR, Dv(D_NORM));
    w.fieldList(hy + "/weightedNeighborSum", name, n, SCALAR, Dv(D_WNS));
    w.fieldList(hy + "/massSecondMoment", name, n, SYMTENSOR, Dv(D_M2));
    w.fieldList(hy + "/XSPHWeightSum", name, n, SCALAR, Dv(D_XSPHW));
    w.fieldList(hy + "/XSPHDeltaV", name, n, VECTOR, Dv(D_XSPHDV));
    const bool one = p.omegaResetByStep;
    w.fieldList(hy + "/omegaGradh", name, n, SCALAR, [&h, one](int64_t i, int) { return one ? 1.0 : h.s(S_OMEGA, i); });
    w.fieldList(hy + "/DxDt", name, n, VECTOR, Dv(D_DXDT));
    w.fieldList(hy + "/DvDt", name, n, VECTOR, Dv(D_DVDT));
    w.fieldList(hy + "/DmassDensityDt", name, n, SCALAR, Dv(D_DRHODT));
    w.fieldList(hy + "/DspecificThermalEnergyDt", name, n, SCALAR, Dv(D_DEPSDT));
    w.fieldList(hy + "/DHDt", name, n, SYMTENSOR, Dv(D_DHDT));
    w.fieldList(hy + "/DvDx", name, n, TENSOR, Dv(D_DVDX));
    w.fieldList(hy + "/internalDvDx", name, n, TENSOR, Dv(D_DVDX));
    w.fieldList(hy + "/maxViscousPressure", name, n, SCALAR, Dv(D_MAXVP));
    w.fieldList(hy + "/effectiveViscousPressure", name, n, SCALAR, Dv(D_EFFVP));
    w.fieldList(hy + "/massDensityCorrection", name, n, SCALAR, constant(0.0));
    w.fieldList(hy + "/viscousWork", name, n, SCALAR, Dv(D_VISCW));
    w.fieldList(hy + "/M", name, n, TENSOR, Dv(D_M));
    w.fieldList(hy + "/localM", name, n, TENSOR, Dv(D_M));
  } else {
    w.fieldList(hy + "/specificThermalEnergy0", name, n, SCALAR, eps0);
    w.fieldList(hy + "/entropy", name, n, SCALAR, entropy);
    w.fieldList(hy + "/Hideal", name, n, SYMTENSOR, Dv(D_HIDEAL));
    w.fieldList(hy + "/maxViscousPressure", name, n, SCALAR, Dv(D_MAXVP));
    w.fieldList(hy + "/effViscousPressure", name, n, SCALAR, Dv(D_EFFVP));
    w.fieldList(hy + "/viscousWork", name, n, SCALAR, Dv(D_VISCW));
    w.fieldList(hy + "/weightedNeighborSum", name, n, SCALAR, Dv(D_WNS));
    w.fieldList(hy + "/massSecondMoment", name, n, SYMTENSOR, Dv(D_M2));
    w.fieldList(hy + "/XSPHDeltaV", name, n, VECTOR, Dv(D_XSPHDV));
    w.fieldList(hy + "/DxDt", name, n, VECTOR, Dv(D_DXDT));
    w.fieldList(hy + "/DvDt", name, n, VECTOR, Dv(D_DVDT));
    w.fieldList(hy + "/DmassDensityDt", name, n, SCALAR, Dv(D_DRHODT));
    w.fieldList(hy + "/DspecificThermalEnergyDt", name, n, SCALAR, Dv(D_DEPSDT));
    w.fieldList(hy + "/DHDt", name, n, SYMTENSOR, Dv(D_DHDT));
    w.fieldList(hy + "/DvDx", name, n, TENSOR, Dv(D_DVDX));
    w.fieldList(hy + "/internalDvDx", name, n, TENSOR, Dv(D_DVDX));
    w.fieldList(hy + "/Volume", name, n, SCALAR, S(S_VOL));
    w.fieldList(hy + "/massDensityGradient", name, n, VECTOR, Kv(K_GRADRHO));
    w.fieldList(hy + "/A", name, n, SCALAR, Kh(K_A));
    w.fieldList(hy + "/B", name, n, VECTOR, Kh(K_B));
    w.emptyFieldList(hy + "/C");
    w.fieldList(hy + "/gradA", name, n, VECTOR, Kh(K_GRADA));
    w.fieldList(hy + "/gradB", name, n, TENSOR, Kh(K_GRADB));
    w.emptyFieldList(hy + "/gradC");
    w.fieldList(hy + "/surfacePoint", name, n, INTEGER, constant(0.0));
  }

  // the periodic boundaries: PeriodicBoundary(plane at xmin facing +e, plane
  // at xmax facing -e) and its two planar boundaries, entering at each plane
  size_t l = 3;
  for (int a = 0; a < 3; ++a) {
    if (!c.periodic[a]) continue;
    const double lo[3] = {c.xmin[0], c.xmin[1], c.xmin[2]}, hi[3] = {c.xmax[0], c.xmax[1], c.xmax[2]};
    double up[3] = {0.0, 0.0, 0.0}, down[3] = {0.0, 0.0, 0.0};
    up[a] = 1.0;
    down[a] = -1.0;
    const double* planes[3][4] = {{lo, up, hi, down}, {lo, up, hi, down}, {hi, down, lo, up}};
    for (int k = 0; k < 3; ++k, ++l) {
      w.value(labels[l] + "/enterPlane/point", planes[k][0], 3);
      w.value(labels[l] + "/enterPlane/normal", planes[k][1], 3);
      w.value(labels[l] + "/exitPlane/point", planes[k][2], 3);
      w.value(labels[l] + "/exitPlane/normal", planes[k][3], 3);
    }
  }

  // the integrator
  const std::string in = labels[l];
  w.value(in + "/lastDt", p.lastDt);
  w.value(in + "/currentTime", p.time);
  w.value(in + "/currentCycle", (long long)p.cycle);
  if (!w.ok()) { set_error("restart file write failed"); return SPHGPU_ERR_ARG; }
  return SPHGPU_OK;
}

// ---- reader

class FlatReader {
 public:
  int load(const char* path) {
    FILE* f = std::fopen(path, "rb");
    if (!f) { set_error(std::string("cannot open restart file: ") + std::strerror(errno)); return SPHGPU_ERR_ARG; }
    char buf[1 << 16];
    size_t k;
    while ((k = std::fread(buf, 1, sizeof(buf), f)) > 0) text_.append(buf, k);
    std::fclose(f);
    lines_.push_back(0);
    for (size_t i = 0; i < text_.size(); ++i)
      if (text_[i] == '\n' && i + 1 < text_.size()) lines_.push_back(i + 1);
    return SPHGPU_OK;
  }
  // FlatFileIO::findPathName: the first line whose first |path| characters
  // are the path; the position after them, or npos.
  size_t find(const std::string& path) const {
    for (size_t s : lines_)
      if (text_.compare(s, path.size(), path) == 0) return s + path.size();
    return std::string::npos;
  }
  // the rest of the line after the path's separating blank (operator>>
  // of a string reads a line and drops that blank)
  bool line(const std::string& path, std::string& out) const {
    size_t s = find(path);
    if (s == std::string::npos) return missing(path);
    const size_t e = text_.find('\n', s);
    out = text_.substr(s, (e == std::string::npos ? text_.size() : e) - s);
    if (!out.empty()) out.erase(0, 1);
    return true;
  }
  // numbers after the path; "(" and ")" are skipped
  bool numbers(const std::string& path, size_t count, std::vector<double>& out) const {
    size_t s = find(path);
    if (s == std::string::npos) return missing(path);
    out.clear();
    const char* p = text_.c_str() + s;
    const char* end = text_.c_str() + text_.size();
    while (out.size() < count && p < end) {
      while (p < end && (*p == ' ' || *p == '\n' || *p == '\t' || *p == '\r')) ++p;
      if (p < end && (*p == '(' || *p == ')')) { ++p; continue; }
      char* q = nullptr;
      const double v = std::strtod(p, &q);
      if (q == p) break;
      out.push_back(v);
      p = q;
    }
    if (out.size() != count) { set_error("restart file: malformed value at " + path); return false; }
    return true;
  }
  // a Field of n internal values with `comps` numbers each
  bool field(const std::string& path, int64_t n, int comps, std::vector<double>& out) const {
    std::vector<double> all;
    if (!numbers(path, 1 + (size_t)n*comps, all)) return false;
    if ((int64_t)all[0] != n) { set_error("restart file: " + path + " holds a different node count"); return false; }
    out.assign(all.begin() + 1, all.end());
    return true;
  }
  // a FieldList of the one NodeList
  bool fieldList(const std::string& path, const std::string& name, int64_t n, int comps,
                 std::vector<double>& out) const {
    std::string names;
    if (!line(path + "/NodeListNames", names)) return false;
    const std::string want = name + "|";
    if (names.compare(0, want.size(), want) != 0 || names.find('|', want.size()) != std::string::npos) {
      set_error("restart file: " + path + " is not a FieldList of the NodeList " + name);
      return false;
    }
    return field(path + "/Field0", n, comps, out);
  }

 private:
  static bool missing(const std::string& path) {
    set_error("restart file: no " + path);
    return false;
  }
  std::string text_;
  std::vector<size_t> lines_;
};

int read_restart(Problem& p, const FlatReader& r, HostState& h) {
  const sphgpu_config& c = p.cfg;
  const int64_t n = p.n;
  const bool crk = c.hydro == SPHGPU_HYDRO_CRKSPH;
  const std::vector<std::string> labels = restart_labels(c);
  const std::string nl = labels[0], hy = labels[2];
  std::string name, count;
  if (!r.line(nl + "/name", name) || !r.line(nl + "/numNodes", count)) return SPHGPU_ERR_ARG;
  if (std::strtoll(count.c_str(), nullptr, 10) != n) {
    set_error("restart file holds " + count + " nodes, the problem " + std::to_string(n));
    return SPHGPU_ERR_ARG;
  }
  std::vector<double> v;
  // into column f0.. of an SoA block
  auto put = [n](std::vector<double>& dst, int f0, int comps, const std::vector<double>& src) {
    for (int64_t i = 0; i < n; ++i)
      for (int k = 0; k < comps; ++k) dst[(f0 + k)*n + i] = src[i*comps + k];
  };
  struct Item { const char* key; bool list; int block; int f0; int comps; };
  // block 0 = S, 1 = S0, 2 = D, 3 = K
  std::vector<Item> items = {
      {"/mass", false, 0, S_M, 1}, {"/positions", false, 0, S_X, 3}, {"/velocity", false, 0, S_VX, 3},
      {"/H", false, 0, S_H, 6}, {"/massDensity", false, 0, S_RHO, 1},
      {"/specificThermalEnergy", false, 0, S_EPS, 1},
  };
  const std::vector<Item> common = {
      {"/pressure", true, 0, S_P, 1}, {"/soundSpeed", true, 0, S_CS, 1},
      {"/specificThermalEnergy0", true, 1, S_EPS, 1}, {"/entropy", true, 1, S0_ENTROPY, 1},
      {"/Hideal", true, 2, D_HIDEAL, 6}, {"/weightedNeighborSum", true, 2, D_WNS, 1},
      {"/massSecondMoment", true, 2, D_M2, 6}, {"/XSPHDeltaV", true, 2, D_XSPHDV, 3},
      {"/DxDt", true, 2, D_DXDT, 3}, {"/DvDt", true, 2, D_DVDT, 3}, {"/DmassDensityDt", true, 2, D_DRHODT, 1},
      {"/DspecificThermalEnergyDt", true, 2, D_DEPSDT, 1}, {"/DHDt", true, 2, D_DHDT, 6},
      {"/DvDx", true, 2, D_DVDX, 9}, {"/maxViscousPressure", true, 2, D_MAXVP, 1},
      {"/viscousWork", true, 2, D_VISCW, 1},
  };
  items.insert(items.end(), common.begin(), common.end());
  if (!crk) {
    const std::vector<Item> sph = {
        {"/massDensitySum", true, 2, D_RHOSUM, 1}, {"/normalization", true, 2, D_NORM, 1},
        {"/XSPHWeightSum", true, 2, D_XSPHW, 1}, {"/omegaGradh", true, 0, S_OMEGA, 1},
        {"/effectiveViscousPressure", true, 2, D_EFFVP, 1}, {"/M", true, 2, D_M, 9},
    };
    items.insert(items.end(), sph.begin(), sph.end());
  } else {
    const std::vector<Item> ck = {
        {"/effViscousPressure", true, 2, D_EFFVP, 1}, {"/Volume", true, 0, S_VOL, 1},
        {"/massDensityGradient", true, 3, K_GRADRHO, 3}, {"/A", true, 3, K_A, 1}, {"/B", true, 3, K_B, 3},
        {"/gradA", true, 3, K_GRADA, 3}, {"/gradB", true, 3, K_GRADB, 9},
    };
    items.insert(items.end(), ck.begin(), ck.end());
  }
  std::vector<double>* blocks[4] = {&h.S, &h.S0, &h.D, &h.K};
  if (crk) h.Kheld.assign((size_t)K_M0*n, 0.0);
  for (const Item& it : items) {
    const bool ok = it.list ? r.fieldList(hy + it.key, name, n, it.comps, v)
                            : r.field(nl + it.key, n, it.comps, v);
    if (!ok) return SPHGPU_ERR_ARG;
    put(*blocks[it.block], it.f0, it.comps, v);
    if (it.block == 3 && it.f0 < K_M0) put(h.Kheld, it.f0, it.comps, v);
  }
  std::vector<double> t;
  const std::string in = labels.back();
  if (!r.numbers(in + "/lastDt", 1, t)) return SPHGPU_ERR_ARG;
  const double lastDt = t[0];
  if (!r.numbers(in + "/currentTime", 1, t)) return SPHGPU_ERR_ARG;
  const double time = t[0];
  if (!r.numbers(in + "/currentCycle", 1, t)) return SPHGPU_ERR_ARG;
  p.lastDt = lastDt;
  p.time = time;
  p.cycle = (int64_t)t[0];
  return SPHGPU_OK;
}

}  // namespace
}  // namespace sphgpu

using namespace sphgpu;

extern "C" {

int sphgpu_restart_labels(const sphgpu_config* cfg, char* buffer, int64_t bytes) {
  if (cfg == nullptr || buffer == nullptr || bytes <= 0) return SPHGPU_ERR_ARG;
  std::string all;
  for (const std::string& l : restart_labels(*cfg)) all += l + "\n";
  if ((int64_t)all.size() + 1 > bytes) { set_error("label buffer too small"); return SPHGPU_ERR_ARG; }
  std::memcpy(buffer, all.c_str(), all.size() + 1);
  return SPHGPU_OK;
}

int sphgpu_restart_dump(sphgpu_problem* p, const char* path, const char* node_list_name) {
  if (p == nullptr || path == nullptr) return SPHGPU_ERR_ARG;
  const std::string name = node_list_name ? node_list_name : "nodes";
  if (name.empty() || name.find('|') != std::string::npos || name.find('\n') != std::string::npos) {
    set_error("NodeList name must be non-empty without '|' or newlines");
    return SPHGPU_ERR_ARG;
  }
  HostState h;
  SPH_TRY(download_state(*p, h));
  FILE* f = std::fopen(path, "wb");
  if (!f) { set_error(std::string("cannot create restart file: ") + std::strerror(errno)); return SPHGPU_ERR_ARG; }
  const int rc = write_restart(*p, h, f, name);
  if (std::fclose(f) != 0 && rc == SPHGPU_OK) { set_error("restart file write failed"); return SPHGPU_ERR_ARG; }
  return rc;
}

int sphgpu_restart_restore(sphgpu_problem* p, const char* path) {
  if (p == nullptr || path == nullptr) return SPHGPU_ERR_ARG;
  FlatReader r;
  SPH_TRY(r.load(path));
  HostState h;
  SPH_TRY(download_state(*p, h));          // columns the file does not carry keep their values
  const bool crkForm = p->cfg.hydro == SPHGPU_HYDRO_CRKSPH;
  // ... or take the reference's defaults where the problem has none yet
  if (!p->haveDerivs) std::fill(h.D.begin(), h.D.end(), 0.0);
  for (int64_t i = 0; i < p->n; ++i) {
    if (crkForm) h.S[S_OMEGA*p->n + i] = 1.0;
    else h.S[S_VOL*p->n + i] = 0.0;
  }
  const double time0 = p->time, lastDt0 = p->lastDt;
  const int64_t cycle0 = p->cycle;
  const int rc = read_restart(*p, r, h);
  if (rc != SPHGPU_OK) {
    p->time = time0; p->lastDt = lastDt0; p->cycle = cycle0;
    return rc;
  }
  const bool crk = p->cfg.hydro == SPHGPU_HYDRO_CRKSPH;
  if (crk && (p->K == nullptr || p->Kheld == nullptr)) {
    if ((p->K == nullptr && dev_alloc(reinterpret_cast<void**>(&p->K), sizeof(double)*NCRK*(size_t)p->n) != cudaSuccess) ||
        (p->Kheld == nullptr &&
         dev_alloc(reinterpret_cast<void**>(&p->Kheld), sizeof(double)*K_M0*(size_t)p->n) != cudaSuccess)) {
      set_error("CRKSPH field allocation failed");
      return SPHGPU_ERR_NOMEM;
    }
  }
  SPH_CHECK(cudaMemcpy(p->S, h.S.data(), sizeof(double)*h.S.size(), cudaMemcpyHostToDevice));
  SPH_CHECK(cudaMemcpy(p->S0, h.S0.data(), sizeof(double)*h.S0.size(), cudaMemcpyHostToDevice));
  SPH_CHECK(cudaMemcpy(p->D, h.D.data(), sizeof(double)*h.D.size(), cudaMemcpyHostToDevice));
  if (crk) {
    SPH_CHECK(cudaMemcpy(p->K, h.K.data(), sizeof(double)*h.K.size(), cudaMemcpyHostToDevice));
    SPH_CHECK(cudaMemcpy(p->Kheld, h.Kheld.data(), sizeof(double)*h.Kheld.size(), cudaMemcpyHostToDevice));
  }
  SPH_CHECK(cudaMemcpy(p->d_scal + SC_LASTDT, &p->lastDt, sizeof(double), cudaMemcpyHostToDevice));
  p->haveNbrs = false;
  p->haveDerivs = true;
  p->crkVolumeReady = crk;
  p->omegaResetByStep = false;
  return SPHGPU_OK;
}

}  // extern "C"
