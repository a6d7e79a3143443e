// gencore.cpp -- DiagnosticCUDA (device sums + host post-processing) and the
// Gencore time-stepping loop, plain (FP64 drop-in) and fused mixed precision.
#include <chrono>
#include <cmath>
#include <algorithm>
#include <cstdio>
#include <cstring>

#include "g4file.h"
#include "g4h_internal.h"
#include "genesis4.h"

namespace g4h {

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

double* slot(std::map<std::string, std::vector<double>>& out, const std::string& key) {
  auto it = out.find(key);
  if (it == out.end() || it->second.empty()) return nullptr;
  return it->second.data();
}

inline void put(double* p, size_t i, double v) {
  if (p) p[i] = v;
}

inline double sqrt_abs(double v) { return std::sqrt(std::fabs(v)); }

const char* kBeamSlice[] = {"energy", "energyspread", "xposition", "xsize", "yposition",
                            "ysize", "pxposition", "pyposition", "current", "emitx",
                            "emity", "betax", "betay", "alphax", "alphay", "bunching",
                            "bunchingphase"};
const char* kBeamAux[] = {"efield", "wakefield", "LSCfield", "SSCfield", "xmin", "xmax",
                          "pxmin", "pxmax", "ymin", "ymax", "pymin", "pymax", "emin", "emax"};
const char* kBeamGlobal[] = {"Global/energy", "Global/energyspread", "Global/xposition",
                             "Global/xsize", "Global/yposition", "Global/ysize"};
const char* kFieldSlice[] = {"power", "xposition", "xsize", "yposition", "ysize",
                             "intensity-nearfield", "phase-nearfield",
                             "intensity-farfield", "phase-farfield"};
const char* kFieldGlobal[] = {"Global/energy", "Global/xposition", "Global/xsize",
                              "Global/yposition", "Global/ysize",
                              "Global/intensity-nearfield", "Global/intensity-farfield"};

}  // namespace

// Record layout of the diagnostics the CUDA calc fills: val[2] beam group,
// val[3 + i] field i, each per-slice record nz * nslice long and each global
// record nz long (src/Core/DiagnosticCUDA.cpp:395-408).
void Diagnostic::init(int nz, int nslice, int nfield, const FilterDiagnostics& f) {
  zout.assign(nz, 0.0);
  val.assign(3 + nfield, {});
  const size_t ns = (size_t)nz * nslice;
  auto& b = val[2];
  for (auto* k : kBeamSlice) b[k].assign(ns, 0.0);
  const int nh = std::max(1, f.beam.harm);
  auto add_harm = [&](int h) {
    b["bunching" + std::to_string(h)].assign(ns, 0.0);
    b["bunchingphase" + std::to_string(h)].assign(ns, 0.0);
  };
  if (f.beam.exclharm && nh > 1)
    add_harm(nh);
  else
    for (int h = 2; h <= nh; ++h) add_harm(h);
  if (f.beam.auxiliar)
    for (auto* k : kBeamAux) b[k].assign(ns, 0.0);
  if (f.beam.global)
    for (auto* k : kBeamGlobal) b[k].assign(nz, 0.0);
  for (int i = 0; i < nfield; ++i) {
    auto& g = val[3 + i];
    for (auto* k : kFieldSlice) g[k].assign(ns, 0.0);
    if (f.field.global)
      for (auto* k : kFieldGlobal) g[k].assign(nz, 0.0);
    g["dgrid"].assign(1, 0.0);
    g["gridspacing"].assign(1, 0.0);
    g["ngrid"].assign(1, 0.0);
  }
}

// Host part of DiagnosticCUDA::calcBeam (src/Core/DiagnosticCUDA.cpp:449-631)
void finish_beam_diag(const FilterDiagnostics& f, int iz, int nslice, int nharm,
                      const double* stats, const double* bre, const double* bim,
                      const std::vector<double>& current, const std::vector<double>& eloss,
                      const std::vector<double>& longESC,
                      std::map<std::string, std::vector<double>>& out) {
  double* p[17];
  for (int k = 0; k < 17; ++k) p[k] = slot(out, kBeamSlice[k]);
  double* aux[14];
  for (int k = 0; k < 14; ++k) aux[k] = slot(out, kBeamAux[k]);
  double* glob[6];
  for (int k = 0; k < 6; ++k) glob[k] = slot(out, kBeamGlobal[k]);
  std::vector<double*> pb(nharm, nullptr), pp(nharm, nullptr);
  pb[0] = p[15];
  pp[0] = p[16];
  for (int ih = 1; ih < nharm; ++ih) {
    if (f.beam.exclharm && ih != nharm - 1) continue;
    pb[ih] = slot(out, "bunching" + std::to_string(ih + 1));
    pp[ih] = slot(out, "bunchingphase" + std::to_string(ih + 1));
  }
  double gc = 0, gg1 = 0, gg2 = 0, gx1 = 0, gx2 = 0, gy1 = 0, gy2 = 0;
  for (int is = 0; is < nslice; ++is) {
    const double* s = stats + 23 * (size_t)is;
    const double nrm = s[12] > 0 ? 1.0 / s[12] : 1.0;
    const double g1 = s[0] * nrm, g2 = s[1] * nrm, x1 = s[2] * nrm, x2 = s[3] * nrm;
    const double y1 = s[4] * nrm, y2 = s[5] * nrm, px1 = s[6] * nrm, px2 = s[7] * nrm;
    const double py1 = s[8] * nrm, py2 = s[9] * nrm, xpx = s[10] * nrm, ypy = s[11] * nrm;
    const size_t idx = (size_t)iz * nslice + is;
    const double cur = is < (int)current.size() ? current[is] : 0.0;
    if (f.beam.energy) {
      put(p[0], idx, g1);
      put(p[1], idx, sqrt_abs(g2 - g1 * g1));
    }
    if (f.beam.spatial) {
      put(p[2], idx, x1);
      put(p[3], idx, sqrt_abs(x2 - x1 * x1));
      put(p[4], idx, y1);
      put(p[5], idx, sqrt_abs(y2 - y1 * y1));
      put(p[6], idx, px1);
      put(p[7], idx, py1);
    }
    for (int ih = 0; ih < nharm; ++ih) {
      if (!pb[ih]) continue;
      const double br = bre[(size_t)is * nharm + ih] * nrm, bi = bim[(size_t)is * nharm + ih] * nrm;
      put(pb[ih], idx, std::hypot(br, bi));
      put(pp[ih], idx, std::atan2(bi, br));
    }
    if (f.beam.auxiliar) {
      const double el = is < (int)eloss.size() ? eloss[is] : 0.0;
      const double sc = is < (int)longESC.size() ? longESC[is] : 0.0;
      put(aux[0], idx, el + sc);
      put(aux[1], idx, el);
      put(aux[2], idx, sc);
      put(aux[3], idx, 0.0);  // BeamSolverCUDA::getSCField: no space charge on device
      for (int k = 0; k < 10; ++k) put(aux[4 + k], idx, s[13 + k]);
    }
    if (f.beam.current || iz == 0) put(p[8], idx, cur);
    if (f.beam.twiss || iz == 0) {
      const double cx = xpx - x1 * px1, cy = ypy - y1 * py1;
      const double ex = std::sqrt(std::fabs((x2 - x1 * x1) * (px2 - px1 * px1) - cx * cx));
      const double ey = std::sqrt(std::fabs((y2 - y1 * y1) * (py2 - py1 * py1) - cy * cy));
      put(p[9], idx, ex);
      put(p[10], idx, ey);
      put(p[11], idx, ex > 0 ? (x2 - x1 * x1) / ex * g1 : 0.0);
      put(p[12], idx, ey > 0 ? (y2 - y1 * y1) / ey * g1 : 0.0);
      put(p[13], idx, ex > 0 ? -cx / ex : 0.0);
      put(p[14], idx, ey > 0 ? -cy / ey : 0.0);
    }
    if (f.beam.global) {
      gc += cur;
      gg1 += cur * g1;
      gg2 += cur * g2;
      gx1 += cur * x1;
      gx2 += cur * x2;
      gy1 += cur * y1;
      gy2 += cur * y2;
    }
  }
  if (f.beam.global) {
    const double nrm = gc > 0 ? 1.0 / gc : 1.0;
    gg1 *= nrm, gg2 *= nrm, gx1 *= nrm, gx2 *= nrm, gy1 *= nrm, gy2 *= nrm;
    if (f.beam.energy) {
      put(glob[0], iz, gg1);
      put(glob[1], iz, sqrt_abs(gg2 - gg1 * gg1));
    }
    if (f.beam.spatial) {
      put(glob[2], iz, gx1);
      put(glob[3], iz, sqrt_abs(gx2 - gx1 * gx1));
      put(glob[4], iz, gy1);
      put(glob[5], iz, sqrt_abs(gy2 - gy1 * gy1));
    }
  }
}

// Host part of DiagnosticCUDA::calcField (src/Core/DiagnosticCUDA.cpp:661-799);
// center holds the centre cell per slice as (re, im) pairs, `stride` doubles
// apart (2 for g4b_diag_field, 9 for the fused run's history).
void finish_field_diag(const FilterDiagnostics& f, int iz, int nslice, int ngrid, double dgrid,
                       double gridmax, double xlambda, double slicelength, const double* stats,
                       int stats_stride, const double* center, int center_stride,
                       std::map<std::string, std::vector<double>>& out) {
  double* p[9];
  for (int k = 0; k < 9; ++k) p[k] = slot(out, kFieldSlice[k]);
  double* glob[7];
  for (int k = 0; k < 7; ++k) glob[k] = slot(out, kFieldGlobal[k]);
  const double ks = 4.0 * std::asin(1.0) / xlambda;
  const double scl = dgrid * eev / ks;
  double gp = 0, gx1 = 0, gx2 = 0, gy1 = 0, gy2 = 0, gff = 0, gin = 0;
  for (int is = 0; is < nslice; ++is) {
    const double* s = stats + (size_t)stats_stride * is;
    const double praw = s[0];
    double x1 = s[1], x2 = s[2], y1 = s[3], y2 = s[4];
    if (f.field.global) {
      gp += praw;
      gx1 += x1;
      gx2 += x2;
      gy1 += y1;
      gy2 += y2;
    }
    if (praw > 0) {
      x1 /= praw;
      x2 /= praw;
      y1 /= praw;
      y2 /= praw;
    }
    x2 = std::sqrt(std::fabs(x2 - x1 * x1));
    y2 = std::sqrt(std::fabs(y2 - y1 * y1));
    const double cre = center[(size_t)center_stride * is], cim = center[(size_t)center_stride * is + 1];
    double inten = cre * cre + cim * cim;
    const double iphi = std::atan2(cim, cre);
    double ff = (s[5] * s[5] + s[6] * s[6]) * dgrid * dgrid;
    const double ffphi = std::atan2(s[6], s[5]);
    if (f.field.global) {
      gff += ff;
      gin += inten;
    }
    const size_t idx = (size_t)iz * nslice + is;
    put(p[0], idx, praw * scl * scl / vacimp);
    if (f.field.spatial) {
      put(p[1], idx, x1 * dgrid);
      put(p[2], idx, x2 * dgrid);
      put(p[3], idx, y1 * dgrid);
      put(p[4], idx, y2 * dgrid);
    }
    if (f.field.intensity) {
      put(p[5], idx, inten * eev * eev / ks / ks / vacimp);
      put(p[6], idx, iphi);
      put(p[7], idx, ff);
      put(p[8], idx, ffphi);
    }
  }
  if (f.field.global) {
    const double nrm = gp > 0 ? 1.0 / gp : 1.0;
    gx1 *= nrm, gx2 *= nrm, gy1 *= nrm, gy2 *= nrm;
    gx2 = std::sqrt(std::fabs(gx2 - gx1 * gx1)) * dgrid;
    gy2 = std::sqrt(std::fabs(gy2 - gy1 * gy1)) * dgrid;
    gx1 *= dgrid;
    gy1 *= dgrid;
    gin /= (double)nslice;
    gff /= (double)nslice;
    put(glob[0], iz, gp * scl * scl / vacimp * slicelength / 299792458.0);
    if (f.field.spatial) {
      put(glob[1], iz, gx1);
      put(glob[2], iz, gx2);
      put(glob[3], iz, gy1);
      put(glob[4], iz, gy2);
    }
    if (f.field.intensity) {
      put(glob[5], iz, gin * eev * eev / ks / ks / vacimp);
      put(glob[6], iz, gff);
    }
  }
  if (iz == 0) {
    put(slot(out, "dgrid"), 0, gridmax);
    put(slot(out, "gridspacing"), 0, dgrid);
    put(slot(out, "ngrid"), 0, (double)ngrid);
  }
}

// DiagnosticCUDA::calc (src/Core/DiagnosticCUDA.cpp:380-411)
bool DiagnosticCUDA::calc(Beam* beam, std::vector<Field*>* field, double z, Diagnostic& diag) {
  if (!beam || !beam->beamSoA || !field) return false;
  for (Field* f : *field)
    if (!f || !f->fieldSoA) return false;
  if (iz_ < (int)diag.zout.size()) diag.zout[iz_] = z;
  if (diag.val.size() > 2) calcBeam(beam, diag.val[2]);
  for (size_t i = 0; i < field->size(); ++i)
    if (3 + i < diag.val.size()) calcField((*field)[i], diag.val[3 + i]);
  ++iz_;
  return true;
}

bool DiagnosticCUDA::calcBeam(Beam* beam, std::map<std::string, std::vector<double>>& out) {
  const int nslice = (int)beam->beam.size();
  const int nharm = std::max(1, filter_.beam.harm);
  std::vector<double> stats((size_t)nslice * 23), bre((size_t)nslice * nharm),
      bim((size_t)nslice * nharm);
  check(g4b_diag_beam(beam->beamSoA, nharm, filter_.beam.auxiliar ? 1 : 0, stats.data(),
                      bre.data(), bim.data()),
        "DiagnosticCUDA::calcBeam");
  finish_beam_diag(filter_, iz_, nslice, nharm, stats.data(), bre.data(), bim.data(),
                   beam->current, beam->eloss, beam->longESC, out);
  return true;
}

bool DiagnosticCUDA::calcField(Field* field, std::map<std::string, std::vector<double>>& out) {
  const int nslice = (int)field->field.size();
  std::vector<double> stats((size_t)nslice * 7), center((size_t)nslice * 2);
  check(g4b_field_set_first(field->fieldSoA, field->first), "DiagnosticCUDA::calcField");
  check(g4b_diag_field(field->fieldSoA, stats.data(), center.data()), "DiagnosticCUDA::calcField");
  finish_field_diag(filter_, iz_, nslice, field->ngrid, field->dgrid, field->gridmax,
                    field->xlambda, field->slicelength, stats.data(), 7, center.data(), 2, out);
  return true;
}

// Gencore::run (src/Core/Gencore.cpp:19-315), use_cuda branch, one rank.
// Step order per lattice step: marker -> Beam::track -> Field::track (every
// field) -> slippage -> diagnostics on output steps.  A marker placed after
// lattice step k acts at the start of step k+1 (the last one after the loop).
bool Gencore::run(Beam* beam, std::vector<Field*>* field, Setup* setup, Undulator* und,
                  bool isTime, bool isScan, bool periodic, bool use_cuda,
                  FilterDiagnostics& filter, Diagnostic& diag, GencoreTimers* timers) {
  if (!use_cuda)
    throw std::runtime_error("Gencore::run: use_cuda=false needs the upstream CPU solvers");
  g4b_ctx* ctx = cuda_context();
  beam->setUseCuda(true);
  beam->pack_beam_to_soa();
  for (Field* f : *field) f->pack_field_to_soa();
  std::string rn, fnbase;
  setup->getRootName(&rn);
  setup->RootName_to_FileName(&fnbase, &rn);
  Control host_control;
  host_control.init(0, 1, fnbase, beam, field, und, isTime, isScan, periodic);
  ControlCUDA control;
  control.init(0, 1, isTime, periodic, beam->slicelength / beam->reflength);
  DiagnosticCUDA dcuda;
  dcuda.init(filter);
  und->reset();
  diag.init(und->outlength(), (int)beam->beam.size(), (int)field->size(), filter);
  dcuda.calc(beam, field, und->getz(), diag);
  GencoreTimers t;
  auto phase = [&](double& acc, auto&& fn) {
    if (timers) g4b_ctx_synchronize(ctx);
    const double t0 = timers ? now_s() : 0.0;
    fn();
    if (timers) {
      check(g4b_ctx_synchronize(ctx), "Gencore::run");
      acc += now_s() - t0;
    }
  };
  while (und->advance(0)) {
    bool error_IO = false;
    control.applyMarker(&host_control, beam, field, und, error_IO);
    if (error_IO) throw std::runtime_error("Gencore::run: marker dump: " + std::string(last_error()));
    const double delz = und->steplength();
    phase(t.beam, [&] { beam->track(delz, field, und); });
    phase(t.field, [&] {
      for (Field* f : *field) f->track(delz, beam, und);
    });
    phase(t.slip, [&] {
      for (Field* f : *field) control.applySlippage(und->slippage(), f);
    });
    phase(t.diag, [&] {
      if (und->outstep()) dcuda.calc(beam, field, und->getz(), diag);
    });
    ++t.steps;
    if (und->steps[und->getStep()].marker & 8) break;  // stop marker
  }
  phase(t.unpack, [&] {
    beam->unpack_soa_to_beam();
    for (Field* f : *field) f->unpack_soa_to_field();
  });
  bool error_IO = false;  // last marker action (src/Core/Gencore.cpp:276-279)
  und->seek(t.steps);      // the marker after the last step taken
  control.applyMarker(&host_control, beam, field, und, error_IO);
  if (error_IO) throw std::runtime_error("Gencore::run: marker dump: " + std::string(last_error()));
  check(g4b_ctx_synchronize(ctx), "Gencore::run");
  if (timers) *timers = t;
  // write out diagnostic arrays (src/Core/Gencore.cpp:297)
  if (!diag.writeToOutputFile(beam, field, setup, und))
    throw std::runtime_error("Gencore::run: output file: " + std::string(last_error()));
  return true;
}

// The records as <fnbase>.out.g4: "Beam/<record>" [nz][nslice] (global
// records [nz]), "Field/<record>" for the first field and "Field<h>/..." for
// a field of harmonic h, "Lattice/zplot" (output positions) and the per-step
// lattice tables "Lattice/{z, dz, aw, ku, kx, ky, qf, cx, cy, chic_angle,
// slippage}", "Meta/{nslice, nfield, steps}".
bool Diagnostic::writeToOutputFile(Beam* beam, std::vector<Field*>* field, Setup* setup,
                                   Undulator* und) {
  std::string rn, fnbase;
  setup->getRootName(&rn);
  setup->RootName_to_FileName(&fnbase, &rn);
  output_file.clear();
  if (fnbase.empty()) return true;
  DataFile f;
  const uint64_t nz = zout.size(), ns = beam->beam.size();
  auto put_group = [&](const std::string& g, const std::map<std::string, std::vector<double>>& m) {
    for (auto& [k, v] : m) {
      if (v.size() == nz * ns && ns > 0)
        f.add(g + "/" + k, {nz, ns}, v);
      else
        f.add(g + "/" + k, {(uint64_t)v.size()}, v);
    }
  };
  if (val.size() > 2) put_group("Beam", val[2]);
  std::map<int, int> seen;
  for (size_t i = 0; i < field->size() && 3 + i < val.size(); ++i) {
    const int h = (*field)[i]->getHarm();
    std::string g = h == 1 ? "Field" : "Field" + std::to_string(h);
    if (seen[h]++) g += "_" + std::to_string(seen[h]);
    put_group(g, val[3 + i]);
  }
  f.add("Lattice/zplot", {nz}, zout);
  const uint64_t nst = und->nstep();
  std::vector<double> z(nst), dz(nst), aw(nst), ku(nst), kx(nst), ky(nst), qf(nst), cx(nst),
      cy(nst), ang(nst), slip(nst);
  for (uint64_t i = 0; i < nst; ++i) {
    const LatticeStep& s = und->steps[i];
    z[i] = s.z, dz[i] = s.st.delz, aw[i] = s.st.aw, ku[i] = s.st.ku, kx[i] = s.st.kx,
    ky[i] = s.st.ky, qf[i] = s.st.qf, cx[i] = s.st.cx, cy[i] = s.st.cy,
    ang[i] = s.st.chic_angle, slip[i] = s.slip;
  }
  const std::pair<const char*, std::vector<double>*> lat[] = {
      {"z", &z}, {"dz", &dz}, {"aw", &aw}, {"ku", &ku}, {"kx", &kx}, {"ky", &ky},
      {"qf", &qf}, {"cx", &cx}, {"cy", &cy}, {"chic_angle", &ang}, {"slippage", &slip}};
  for (auto& [k, v] : lat) f.add(std::string("Lattice/") + k, {nst}, *v);
  f.add_scalar("Meta/nslice", (double)ns);
  f.add_scalar("Meta/nfield", (double)field->size());
  f.add_scalar("Meta/steps", (double)nst);
  const std::string path = fnbase + ".out.g4";
  if (!f.write(path)) return false;
  output_file = path;
  return true;
}

// The same loop as one resident mixed-precision run (g4b_run): the lattice is
// uploaded once, the steps are replayed from a CUDA graph and the per-step
// diagnostic sums are read back from the run's history after the loop.
bool run_mixed(Beam* beam, std::vector<Field*>* field, Setup* setup, Undulator* und,
               bool isTime, bool periodic, FilterDiagnostics& filter, Diagnostic& diag,
               GencoreTimers* timers) {
  const int nslice = (int)beam->beam.size();
  const int nfield = (int)field->size();
  if (nfield < 1 || nfield > 8) throw std::runtime_error("run_mixed: 1..8 fields");
  g4b_run_desc d{};
  d.nslice = nslice;
  d.nfield = nfield;
  for (int i = 0; i < nfield; ++i) {
    Field* f = (*field)[i];
    d.harm[i] = f->getHarm();
    d.ngrid[i] = f->ngrid;
    d.gridmax[i] = f->gridmax;
  }
  d.lambda0 = und->lambda0;
  d.gamma_ref = beam->gamma_ref;
  d.sample = beam->slicelength / beam->reflength;
  d.time_run = isTime ? 1 : 0;
  d.periodic = periodic ? 1 : 0;
  d.nbunch = std::max(1, filter.beam.harm);
  d.precision = G4B_MIXED;
  std::vector<int64_t> off(nslice + 1, 0);
  for (int s = 0; s < nslice; ++s) off[s + 1] = off[s] + (int64_t)beam->beam[s].size();
  g4b_run* run = nullptr;
  check(g4b_run_create(cuda_context(), &d, off.data(), &run), "run_mixed");
  struct Guard {
    g4b_run* r;
    ~Guard() { g4b_run_destroy(r); }
  } guard{run};
  const size_t np = (size_t)off[nslice];
  {
    std::vector<double> x(np), y(np), px(np), py(np), g(np), th(np);
    size_t k = 0;
    for (auto& s : beam->beam)
      for (auto& p : s) {
        x[k] = p.x, y[k] = p.y, px[k] = p.px, py[k] = p.py, g[k] = p.gamma, th[k] = p.theta;
        ++k;
      }
    check(g4b_run_upload_beam(run, x.data(), y.data(), px.data(), py.data(), g.data(), th.data()),
          "run_mixed");
  }
  for (int i = 0; i < nfield; ++i) {
    Field* f = (*field)[i];
    const size_t plane = (size_t)f->ngrid * f->ngrid;
    std::vector<double> cells(2 * plane * nslice);
    for (int s = 0; s < nslice; ++s)
      std::memcpy(cells.data() + 2 * plane * s, f->field[s].data(), 16 * plane);
    check(g4b_run_upload_field(run, i, cells.data(), f->first), "run_mixed");
  }
  check(g4b_run_set_current(run, beam->current.data()), "run_mixed");
  {
    std::vector<double> el(nslice);
    for (int s = 0; s < nslice; ++s) el[s] = -beam->longESC[s] / 511000.0;
    check(g4b_run_set_eloss(run, el.data()), "run_mixed");
  }
  const int nstep = und->nstep();
  std::vector<g4b_step> steps(nstep);
  std::vector<double> fc((size_t)nstep * nfield), slip(nstep);
  int nrun = nstep;
  for (int i = 0; i < nstep; ++i) {
    steps[i] = und->steps[i].st;
    slip[i] = und->steps[i].slip;
    for (int k = 0; k < nfield; ++k) fc[(size_t)i * nfield + k] = und->fc_at(i, d.harm[k]);
    if ((und->steps[i].marker & 8) && nrun == nstep) nrun = i + 1;
  }
  check(g4b_run_set_lattice(run, nstep, steps.data(), fc.data(), slip.data(), 0), "run_mixed");

  // initial diagnostics from the host state (FP64, before any step)
  und->reset();
  diag.init(und->outlength(), nslice, nfield, filter);
  const int nharm = d.nbunch;
  {
    std::vector<double> st((size_t)nslice * 23, 0.0), bre((size_t)nslice * nharm, 0.0),
        bim((size_t)nslice * nharm, 0.0);
    for (int s = 0; s < nslice; ++s) {
      double* o = st.data() + 23 * (size_t)s;
      double mn[5] = {1e5, 1e5, 1e5, 1e5, 1e7}, mx[5] = {-1e5, -1e5, -1e5, -1e5, 1.0};
      for (auto& p : beam->beam[s]) {
        const double v[12] = {p.gamma, p.gamma * p.gamma, p.x, p.x * p.x, p.y, p.y * p.y,
                              p.px, p.px * p.px, p.py, p.py * p.py, p.x * p.px, p.y * p.py};
        for (int k = 0; k < 12; ++k) o[k] += v[k];
        o[12] += 1.0;
        const double q[5] = {p.x, p.px, p.y, p.py, p.gamma};
        for (int k = 0; k < 5; ++k) mn[k] = std::min(mn[k], q[k]), mx[k] = std::max(mx[k], q[k]);
        for (int h = 0; h < nharm; ++h) {
          bre[(size_t)s * nharm + h] += std::cos((h + 1) * p.theta);
          bim[(size_t)s * nharm + h] += std::sin((h + 1) * p.theta);
        }
      }
      for (int k = 0; k < 5; ++k) o[13 + 2 * k] = mn[k], o[14 + 2 * k] = mx[k];
    }
    diag.zout[0] = 0.0;
    finish_beam_diag(filter, 0, nslice, nharm, st.data(), bre.data(), bim.data(),
                     beam->current, beam->eloss, beam->longESC, diag.val[2]);
    for (int i = 0; i < nfield; ++i) {
      Field* f = (*field)[i];
      const int n = f->ngrid;
      std::vector<double> fs((size_t)nslice * 7, 0.0), cen((size_t)nslice * 2);
      for (int s0 = 0; s0 < nslice; ++s0) {
        const int is = (nslice + s0 - f->first) % nslice;
        double* o = fs.data() + 7 * (size_t)is;
        const auto& pl = f->field[s0];
        const double sh = -0.5 * (n - 1);
        for (int iy = 0; iy < n; ++iy)
          for (int ix = 0; ix < n; ++ix) {
            const auto c = pl[(size_t)iy * n + ix];
            const double w = std::norm(c), dx = ix + sh, dy = iy + sh;
            o[0] += w, o[1] += dx * w, o[2] += dx * dx * w, o[3] += dy * w, o[4] += dy * dy * w;
            o[5] += c.real(), o[6] += c.imag();
          }
        const auto cc = pl[((size_t)n * n - 1) / 2];
        cen[2 * is] = cc.real(), cen[2 * is + 1] = cc.imag();
      }
      finish_field_diag(filter, 0, nslice, n, f->dgrid, f->gridmax, f->xlambda, f->slicelength,
                        fs.data(), 7, cen.data(), 2, diag.val[3 + i]);
    }
  }

  // final state (or the state at a dump marker) back into the host objects
  auto pull_state = [&]() {
    std::vector<double> x(np), y(np), px(np), py(np), g(np), th(np);
    check(g4b_run_download_beam(run, x.data(), y.data(), px.data(), py.data(), g.data(),
                                th.data()),
          "run_mixed");
    size_t k = 0;
    for (auto& s : beam->beam)
      for (auto& p : s) {
        p.x = x[k], p.y = y[k], p.px = px[k], p.py = py[k], p.gamma = g[k], p.theta = th[k];
        ++k;
      }
    for (int i = 0; i < nfield; ++i) {
      Field* f = (*field)[i];
      const size_t plane = (size_t)f->ngrid * f->ngrid;
      std::vector<double> cells(2 * plane * nslice);
      check(g4b_run_download_field(run, i, cells.data(), &f->first), "run_mixed");
      for (int s = 0; s < nslice; ++s)
        std::memcpy(f->field[s].data(), cells.data() + 2 * plane * s, 16 * plane);
    }
  };
  std::string rn, fnbase;
  setup->getRootName(&rn);
  setup->RootName_to_FileName(&fnbase, &rn);
  Control host_control;
  host_control.init(0, 1, fnbase, beam, field, und, isTime, false, periodic);
  auto marker = [&](int steps_taken) {
    und->seek(steps_taken);
    bool error_IO = false;
    host_control.applyMarker(beam, field, und, error_IO);
    if (error_IO) throw std::runtime_error("run_mixed: marker dump: " + std::string(last_error()));
  };
  // the loop stops where a dump marker acts, to bring the state to the host
  std::vector<int> cuts;
  if (!fnbase.empty())
    for (int i = 0; i + 1 < nrun; ++i)
      if (und->steps[i].marker & 3) cuts.push_back(i + 1);
  cuts.push_back(nrun);
  g4b_ctx* ctx = cuda_context();
  double loop_s = 0.0;
  int done = 0;
  for (int c : cuts) {
    check(g4b_ctx_synchronize(ctx), "run_mixed");
    const double t0 = now_s();
    if (c > done) check(g4b_run_advance(run, done, c - done, 1), "run_mixed");
    check(g4b_ctx_synchronize(ctx), "run_mixed");
    loop_s += now_s() - t0;
    done = c;
    if (c < nrun) {
      pull_state();
      marker(c);
    }
  }

  const size_t rec = 23 + 2 * (size_t)nharm;
  std::vector<double> hb((size_t)nslice * rec), hf((size_t)nfield * nslice * 9);
  std::vector<double> st((size_t)nslice * 23), bre((size_t)nslice * nharm), bim((size_t)nslice * nharm);
  int iz = 1;
  for (int i = 0; i < nrun; ++i) {
    if (!(((i + 1) % und->output_step) == 0 || i + 1 == nstep)) continue;
    check(g4b_run_history(run, i, hb.data(), hf.data()), "run_mixed");
    for (int s = 0; s < nslice; ++s) {
      std::memcpy(st.data() + 23 * (size_t)s, hb.data() + rec * s, 23 * 8);
      for (int h = 0; h < nharm; ++h) {
        bre[(size_t)s * nharm + h] = hb[rec * s + 23 + 2 * h];
        bim[(size_t)s * nharm + h] = hb[rec * s + 24 + 2 * h];
      }
    }
    if (iz < (int)diag.zout.size()) diag.zout[iz] = und->steps[i].z;
    finish_beam_diag(filter, iz, nslice, nharm, st.data(), bre.data(), bim.data(), beam->current,
                     beam->eloss, beam->longESC, diag.val[2]);
    for (int k = 0; k < nfield; ++k) {
      Field* f = (*field)[k];
      const double* rec_f = hf.data() + (size_t)k * nslice * 9;
      finish_field_diag(filter, iz, nslice, f->ngrid, f->dgrid, f->gridmax, f->xlambda,
                        f->slicelength, rec_f, 9, rec_f + 7, 9, diag.val[3 + k]);
    }
    ++iz;
  }
  pull_state();
  marker(nrun);  // the last marker action (src/Core/Gencore.cpp:276-279)
  if (timers) {
    *timers = GencoreTimers{};
    timers->beam = loop_s;  // the fused loop (without the dump stops)
    timers->steps = nrun;
  }
  if (!diag.writeToOutputFile(beam, field, setup, und))
    throw std::runtime_error("run_mixed: output file: " + std::string(last_error()));
  return true;
}

}  // namespace g4h
