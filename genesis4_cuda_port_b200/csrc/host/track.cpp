// track.cpp -- input decks (.in namelists) and the Track driver.
//
// A deck is a sequence of `&group key=value ... &end` blocks, read in order
// as upstream GENESIS 1.3 v4 does: &setup, &lattice, &time, &field (one per
// harmonic), &beam, &efield, &track.  The keys follow the upstream manual; &track
// keeps the reference's keys (src/Main/Track.cpp:8-96, incl. use_cuda and
// low_memory_adisolver) and adds `precision = fp64 | mixed`, which selects
// between the drop-in FP64 classes and the fused mixed-precision run.
// Unknown keys are an error, as in Track::init (src/Main/Track.cpp:98-104).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <sstream>

#include "g4h.h"
#include "g4h_internal.h"
#include "genesis4.h"

namespace g4h {

namespace {

using Group = std::map<std::string, std::string>;

std::string lower(std::string s) {
  for (auto& c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

std::string trim(const std::string& s) {
  size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
  return a == std::string::npos ? "" : s.substr(a, b - a + 1);
}

bool atob(const std::string& v) {
  const std::string s = lower(trim(v));
  return s == "1" || s == "true" || s == "t";
}

// Splits the deck into (group name, key -> value) blocks in file order.
bool parse_namelists(const std::string& text, std::vector<std::pair<std::string, Group>>& out) {
  std::istringstream is(text);
  std::string line;
  bool open = false;
  int lineno = 0;
  while (std::getline(is, line)) {
    ++lineno;
    const auto h = line.find('#');
    if (h != std::string::npos) line = line.substr(0, h);
    line = trim(line);
    if (line.empty()) continue;
    if (line[0] == '&') {
      const std::string name = lower(trim(line.substr(1)));
      if (name == "end") {
        if (!open) {
          set_error("deck: &end without a group at line " + std::to_string(lineno));
          return false;
        }
        open = false;
        continue;
      }
      if (open) {
        set_error("deck: group &" + out.back().first + " not closed before line " +
                  std::to_string(lineno));
        return false;
      }
      out.push_back({name, {}});
      open = true;
      continue;
    }
    if (!open) {
      set_error("deck: text outside a group at line " + std::to_string(lineno));
      return false;
    }
    const auto eq = line.find('=');
    if (eq == std::string::npos) {
      set_error("deck: expected key = value at line " + std::to_string(lineno));
      return false;
    }
    std::string val = trim(line.substr(eq + 1));
    if (!val.empty() && (val.front() == '"' || val.front() == '\'')) val = val.substr(1);
    if (!val.empty() && (val.back() == '"' || val.back() == '\'')) val.pop_back();
    out.back().second[lower(trim(line.substr(0, eq)))] = val;
  }
  if (open) {
    set_error("deck: group &" + out.back().first + " not closed by &end");
    return false;
  }
  return true;
}

// Reads the known keys of one group; anything left is an error.
struct Reader {
  Group g;
  std::string name;
  double num(const char* k, double def) {
    auto it = g.find(k);
    if (it == g.end()) return def;
    const double v = std::atof(it->second.c_str());
    g.erase(it);
    return v;
  }
  bool flag(const char* k, bool def) {
    auto it = g.find(k);
    if (it == g.end()) return def;
    const bool v = atob(it->second);
    g.erase(it);
    return v;
  }
  std::string str(const char* k, const std::string& def) {
    auto it = g.find(k);
    if (it == g.end()) return def;
    const std::string v = it->second;
    g.erase(it);
    return v;
  }
  bool has(const char* k) const { return g.count(k) != 0; }
  bool done() {
    if (g.empty()) return true;
    std::string keys;
    for (auto& kv : g) keys += " " + kv.first;
    set_error("deck: unknown or unsupported keys in &" + name + ":" + keys);
    return false;
  }
};

// Matched Twiss parameters of the periodic cell [0, zmatch): the product of
// the per-step thick-lens maps of the on-axis reference particle (the maps
// TrackBeamCUDA applies, src/Core/TrackBeamCUDA.cpp:27-59,156-180).
bool match_twiss(const Undulator& und, double zmatch, double gamma0, double tw[4]) {
  double m[2][2][2] = {{{1, 0}, {0, 1}}, {{1, 0}, {0, 1}}};
  for (const LatticeStep& ls : und.steps) {
    if (ls.z > zmatch + 1e-9) break;
    const g4b_step& st = ls.st;
    const double aw = st.aw;
    const double bp = std::sqrt(1 - (1 + aw * aw) / gamma0 / gamma0);
    const double quad = st.qf * gamma0;
    const double q[2] = {quad + st.kx * aw * aw / gamma0 / bp, -quad + st.ky * aw * aw / gamma0 / bp};
    const double gz = std::sqrt(gamma0 * gamma0 - 1 - aw * aw);
    for (int p = 0; p < 2; ++p) {
      const double k = q[p] / gz, L = st.delz;
      double a[2][2];
      if (k > 0) {
        const double f = std::sqrt(k);
        a[0][0] = std::cos(f * L), a[0][1] = std::sin(f * L) / f;
        a[1][0] = -f * std::sin(f * L), a[1][1] = std::cos(f * L);
      } else if (k < 0) {
        const double f = std::sqrt(-k);
        a[0][0] = std::cosh(f * L), a[0][1] = std::sinh(f * L) / f;
        a[1][0] = f * std::sinh(f * L), a[1][1] = std::cosh(f * L);
      } else {
        a[0][0] = 1, a[0][1] = L, a[1][0] = 0, a[1][1] = 1;
      }
      double r[2][2];
      for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) r[i][j] = a[i][0] * m[p][0][j] + a[i][1] * m[p][1][j];
      std::memcpy(m[p], r, sizeof r);
    }
  }
  for (int p = 0; p < 2; ++p) {
    const double c = 0.5 * (m[p][0][0] + m[p][1][1]);
    if (std::fabs(c) >= 1.0) {
      set_error("deck: &lattice zmatch: the cell has no periodic (matched) solution");
      return false;
    }
    const double s = (m[p][0][1] >= 0 ? 1.0 : -1.0) * std::sqrt(1 - c * c);
    tw[2 * p] = m[p][0][1] / s;                          // beta
    tw[2 * p + 1] = (m[p][0][0] - m[p][1][1]) / (2 * s);  // alpha
  }
  return true;
}

std::string read_file(const std::string& path) {
  std::ifstream f(path);
  if (!f) return std::string();
  std::stringstream ss;
  ss << f.rdbuf();
  return ss.str();
}

}  // namespace

// Everything a deck defines, resolved to the sizes the run needs.
struct Deck {
  // &setup
  std::string rootname = "genesis", latfile, beamline;
  double gamma0 = 11350.3, lambda0 = 1e-10, delz = 0.015;
  uint64_t seed = 123456789;
  int npart = 8192, nbins = 4;
  bool shotnoise = true, beam_global = true, field_global = true;
  FilterDiagnostics filter;
  // &lattice
  double zmatch = 0;
  // &time
  bool time = false;
  double s0 = 0, slen = 0, sample = 1;
  int nslice = 1;
  // &field (one per harmonic)
  struct FieldIn {
    int harm = 1, ngrid = 151;
    double power = 0, phase = 0, waist = 100e-6, gridmax = 1e-3;
  };
  std::vector<FieldIn> fields;
  // &beam
  g4h_beam_spec beam{};
  double current = 1000;
  // &track
  bool use_cuda = true, low_memory = false, periodic = false;
  bool fft = false, src_filter = false;          // &track fft_fieldsolver, source_filter
  double xcut = 1, ycut = 1, sigmoid = 1;        // &track xcut, ycut, sigmoid
  int precision = G4B_FP64, output_step = 1, beam_dump = 0, field_dump = 0;
  double zstop = 1e9;
  // &efield: short-range space charge (upstream manual keys)
  double sc_rmax = 0;
  int sc_ngrid = 100, sc_nz = 0, sc_nphi = 0;
  Undulator und;
  // files: the deck's directory, &setup outputdir, &importbeam / &importfield
  std::string base, outputdir, import_beam;
  struct ImportField {
    std::string file;
    int harm = 1;
  };
  std::vector<ImportField> import_fields;
};

// a deck's file name, relative to the deck's directory unless absolute
std::string deck_path(const std::string& base, const std::string& f) {
  if (f.empty() || f[0] == '/' || base.empty()) return f;
  return base + "/" + f;
}

bool parse_deck(const std::string& text, const std::string* lat_text, const std::string& base,
                Deck& d) {
  std::vector<std::pair<std::string, Group>> groups;
  if (!parse_namelists(text, groups)) return false;
  bool have_setup = false, have_beam = false, have_track = false;
  bool beam_twiss_set[4] = {false, false, false, false};
  std::string lattice_text;
  for (auto& [name, g] : groups) {
    Reader r{g, name};
    if (name == "setup") {
      have_setup = true;
      d.rootname = r.str("rootname", d.rootname);
      d.outputdir = r.str("outputdir", "");
      d.latfile = r.str("lattice", "");
      d.beamline = r.str("beamline", "");
      d.gamma0 = r.num("gamma0", d.gamma0);
      d.lambda0 = r.num("lambda0", d.lambda0);
      d.delz = r.num("delz", d.delz);
      d.seed = (uint64_t)r.num("seed", (double)d.seed);
      d.npart = (int)r.num("npart", d.npart);
      d.nbins = (int)r.num("nbins", d.nbins);
      d.shotnoise = r.flag("shotnoise", true);
      d.beam_global = r.flag("beam_global_stat", true);
      d.field_global = r.flag("field_global_stat", true);
      d.filter.field.spatial = !r.flag("exclude_spatial_output", false);
      d.filter.beam.spatial = d.filter.field.spatial;
      d.filter.field.intensity = !r.flag("exclude_intensity_output", false);
      d.filter.beam.energy = !r.flag("exclude_energy_output", false);
      d.filter.beam.auxiliar = !r.flag("exclude_aux_output", false);
      d.filter.beam.current = !r.flag("exclude_current_output", false);
      d.filter.beam.twiss = !r.flag("exclude_twiss_output", false);
      if (r.flag("one4one", false)) {
        set_error("deck: one4one = true is not supported (quiet-start beams only)");
        return false;
      }
      if (!r.done()) return false;
      if (d.beamline.empty() || (d.latfile.empty() && !lat_text)) {
        set_error("deck: &setup needs lattice and beamline");
        return false;
      }
      lattice_text = lat_text ? *lat_text : read_file(base.empty() ? d.latfile : base + "/" + d.latfile);
      if (lattice_text.empty()) {
        set_error("deck: cannot read lattice file " + d.latfile);
        return false;
      }
      d.beam.gamma0 = d.gamma0;
      d.beam.delgam = 0.5;
      d.beam.ex = d.beam.ey = 0.3e-6;
      d.beam.betax = d.beam.betay = 15.0;
    } else if (!have_setup) {
      set_error("deck: &" + name + " before &setup");
      return false;
    } else if (name == "lattice") {
      d.zmatch = r.num("zmatch", 0.0);
      if (!r.done()) return false;
    } else if (name == "time") {
      d.time = r.flag("time", true);
      d.s0 = r.num("s0", 0.0);
      d.slen = r.num("slen", 0.0);
      d.sample = r.num("sample", 1.0);
      if (!r.done()) return false;
      if (!(d.sample >= 1)) {
        set_error("deck: &time sample must be >= 1");
        return false;
      }
    } else if (name == "field") {
      Deck::FieldIn f;
      f.harm = (int)r.num("harm", 1);
      f.power = r.num("power", 0.0);
      f.phase = r.num("phase", 0.0);
      f.waist = r.num("waist_size", 100e-6);
      f.gridmax = r.num("dgrid", 1e-3);
      f.ngrid = (int)r.num("ngrid", 151);
      const double lam = r.num("lambda", d.lambda0);
      const double wpos = r.num("waist_pos", 0.0), xc = r.num("xcenter", 0.0),
                   yc = r.num("ycenter", 0.0), xa = r.num("xangle", 0.0), ya = r.num("yangle", 0.0);
      if (!r.done()) return false;
      if (wpos != 0 || xc != 0 || yc != 0 || xa != 0 || ya != 0 ||
          std::fabs(lam - d.lambda0) > 1e-12 * d.lambda0) {
        set_error("deck: &field supports an on-axis Gaussian waist at z = 0 at lambda0 only");
        return false;
      }
      if (f.harm < 1 || f.ngrid < 3) {
        set_error("deck: &field needs harm >= 1 and ngrid >= 3");
        return false;
      }
      d.fields.push_back(f);
    } else if (name == "importbeam") {  // upstream &importbeam: a particle dump
      d.import_beam = deck_path(base, r.str("file", ""));
      r.flag("time", true);
      if (!r.done()) return false;
      if (d.import_beam.empty()) {
        set_error("deck: &importbeam needs file");
        return false;
      }
    } else if (name == "importfield") {  // upstream &importfield: a field dump
      Deck::ImportField fi;
      fi.file = deck_path(base, r.str("file", ""));
      fi.harm = (int)r.num("harmonic", 1);
      r.flag("time", true);
      if (!r.done()) return false;
      if (fi.file.empty()) {
        set_error("deck: &importfield needs file");
        return false;
      }
      d.import_fields.push_back(fi);
    } else if (name == "beam") {
      have_beam = true;
      g4h_beam_spec& b = d.beam;
      b.gamma0 = r.num("gamma", d.gamma0);
      b.delgam = r.num("delgam", b.delgam);
      d.current = r.num("current", d.current);
      b.ex = r.num("ex", b.ex);
      b.ey = r.num("ey", b.ey);
      const char* tk[4] = {"betax", "alphax", "betay", "alphay"};
      double* tv[4] = {&b.betax, &b.alphax, &b.betay, &b.alphay};
      for (int k = 0; k < 4; ++k)
        if (r.has(tk[k])) {
          *tv[k] = r.num(tk[k], 0.0);
          beam_twiss_set[k] = true;
        }
      b.xcenter = r.num("xcenter", 0.0);
      b.ycenter = r.num("ycenter", 0.0);
      b.pxcenter = r.num("pxcenter", 0.0);
      b.pycenter = r.num("pycenter", 0.0);
      if (r.num("bunch", 0.0) != 0 || r.num("emod", 0.0) != 0) {
        set_error("deck: &beam bunch/emod modulation is not supported");
        return false;
      }
      r.num("bunchphase", 0.0);
      r.num("emodphase", 0.0);
      if (!r.done()) return false;
    } else if (name == "efield") {
      d.sc_rmax = r.num("rmax", 0.0);
      d.sc_ngrid = (int)r.num("ngrid", 100);
      d.sc_nz = (int)r.num("nz", 0);
      d.sc_nphi = (int)r.num("nphi", 0);
      const bool longrange = r.flag("longrange", false);
      if (!r.done()) return false;
      if (longrange) {
        set_error("deck: &efield longrange (upstream's long-range model) is not supported");
        return false;
      }
      if (d.sc_rmax < 0 || d.sc_ngrid < 0 || d.sc_nz < 0 || d.sc_nphi < 0) {
        set_error("deck: &efield needs rmax, ngrid, nz, nphi >= 0");
        return false;
      }
    } else if (name == "track") {
      have_track = true;
      d.zstop = r.num("zstop", 1e9);
      d.output_step = std::max(1, (int)r.num("output_step", 1));
      d.field_dump = (int)r.num("field_dump_step", 0);
      d.beam_dump = (int)r.num("beam_dump_step", 0);
      const int sort_step = (int)r.num("sort_step", 0);
      d.filter.beam.harm = std::max(1, (int)r.num("bunchharm", 1));
      d.filter.beam.exclharm = r.flag("exclusive_harmonics", false);
      d.periodic = r.flag("periodic", false);
      d.use_cuda = r.flag("use_cuda", true);
      d.low_memory = r.flag("low_memory_adisolver", false);
      d.fft = r.flag("fft_fieldsolver", false);
      d.src_filter = r.flag("source_filter", false);
      d.xcut = r.num("xcut", 1);
      d.ycut = r.num("ycut", 1);
      d.sigmoid = r.num("sigmoid", 1);
      if (r.has("s0")) d.s0 = r.num("s0", 0.0);
      if (r.has("slen")) d.slen = r.num("slen", 0.0);
      const std::string prec = lower(r.str("precision", "fp64"));
      if (!r.done()) return false;
      if (prec == "fp64")
        d.precision = G4B_FP64;
      else if (prec == "mixed")
        d.precision = G4B_MIXED;
      else {
        set_error("deck: &track precision must be fp64 or mixed");
        return false;
      }
      if (d.fft && d.precision == G4B_MIXED) {
        set_error("deck: fft_fieldsolver runs the FP64 drop-in form (precision = fp64)");
        return false;
      }
      if (d.sc_nz > 0 && d.sc_rmax > 0 && d.precision == G4B_MIXED) {
        set_error("deck: &efield space charge runs the FP64 drop-in form (precision = fp64)");
        return false;
      }
      if (sort_step != 0) {
        set_error("deck: sort_step is not supported");
        return false;
      }
      if (!d.use_cuda) {
        set_error("deck: use_cuda = false selects the upstream CPU path, not in this build");
        return false;
      }
      break;  // one &track per deck is run
    } else {
      set_error("deck: unsupported group &" + name);
      return false;
    }
  }
  if (!have_setup || !have_beam || !have_track || d.fields.empty()) {
    set_error("deck: needs &setup, &field, &beam and &track");
    return false;
  }
  // &time: slices at sample*lambda0 spacing over the window
  d.nslice = d.time ? std::max(1, (int)std::lround(d.slen / (d.sample * d.lambda0))) : 1;
  if (!d.time) d.sample = 1;
  // lattice at the beam energy
  if (!build_lattice(lattice_text, d.beamline, d.delz, d.gamma0, d.lambda0, d.und)) return false;
  if (d.zmatch > 0) {
    double tw[4];
    if (!match_twiss(d.und, d.zmatch, d.beam.gamma0, tw)) return false;
    double* tv[4] = {&d.beam.betax, &d.beam.alphax, &d.beam.betay, &d.beam.alphay};
    for (int k = 0; k < 4; ++k)
      if (!beam_twiss_set[k]) *tv[k] = tw[k];
  }
  // Undulator::updateMarker / updateOutput (src/Main/Track.cpp:134-137)
  d.und.output_step = d.output_step;
  for (int i = 0; i < d.und.nstep(); ++i) {
    LatticeStep& s = d.und.steps[i];
    if (d.field_dump > 0 && (i + 1) % d.field_dump == 0) s.marker |= 2;
    if (d.beam_dump > 0 && (i + 1) % d.beam_dump == 0) s.marker |= 1;
    if (s.z >= d.zstop - 1e-12) {
      s.marker |= 8;
      break;
    }
  }
  // steady state: no global statistics (src/Main/Track.cpp:142-153)
  const bool ssrun = d.nslice == 1;
  d.filter.beam.global = !ssrun && d.beam_global;
  d.filter.field.global = !ssrun && d.field_global;
  d.beam.nslice = d.nslice;
  d.beam.npart = d.npart;
  d.beam.nbins = d.nbins;
  d.beam.shotnoise = d.shotnoise ? 1 : 0;
  d.beam.seed = d.seed;
  d.beam.reflength = d.lambda0;
  d.beam.slicelength = d.lambda0 * d.sample;
  d.base = base;
  for (auto& fi : d.import_fields) {
    bool found = false;
    for (auto& f : d.fields) found |= f.harm == fi.harm;
    if (!found) {
      set_error("deck: &importfield harmonic " + std::to_string(fi.harm) +
                " has no &field of that harmonic");
      return false;
    }
  }
  return true;
}

}  // namespace g4h

using namespace g4h;

struct g4h_deck {
  Deck d;
};

struct g4h_result {
  Diagnostic diag;
  std::string output_file;
  int nslice = 0, nfield = 0, nsteps = 0;
  double seconds = 0;
  std::vector<std::vector<double>> field_out;  // final cells per field
  std::vector<int> first;
};

namespace {

int deck_error(int rc = G4B_ERR_ARG) { return rc; }

bool load_deck(const char* text, const char* lat, const char* base, g4h_deck** out) {
  if (!text || !out) {
    set_error("g4h_deck_parse: null argument");
    return false;
  }
  auto dk = std::make_unique<g4h_deck>();
  const std::string lt = lat ? lat : "";
  if (!parse_deck(text, lat ? &lt : nullptr, base ? base : "", dk->d)) return false;
  *out = dk.release();
  return true;
}

}  // namespace

extern "C" {

int g4h_deck_parse(const char* deck_text, const char* lattice_text, const char* base_dir,
                   g4h_deck** out) {
  return load_deck(deck_text, lattice_text, base_dir, out) ? G4B_OK : deck_error();
}

int g4h_deck_destroy(g4h_deck* dk) {
  delete dk;
  return G4B_OK;
}

int g4h_deck_info(g4h_deck* dk, g4h_deck_summary* s) {
  if (!dk || !s) {
    set_error("g4h_deck_info: null argument");
    return G4B_ERR_ARG;
  }
  const Deck& d = dk->d;
  std::memset(s, 0, sizeof *s);
  s->nslice = d.nslice;
  s->npart = d.npart;
  s->nstep = d.und.nstep();
  s->nfield = (int)d.fields.size();
  for (int i = 0; i < s->nfield && i < 8; ++i) {
    s->harm[i] = d.fields[i].harm;
    s->ngrid[i] = d.fields[i].ngrid;
    s->gridmax[i] = d.fields[i].gridmax;
  }
  s->lambda0 = d.lambda0;
  s->gamma0 = d.gamma0;
  s->sample = d.sample;
  s->time_run = d.time ? 1 : 0;
  s->periodic = d.periodic ? 1 : 0;
  s->precision = d.precision;
  s->low_memory = d.low_memory ? 1 : 0;
  s->output_step = d.output_step;
  s->nout = d.und.outlength();
  s->bunchharm = d.filter.beam.harm;
  s->betax = d.beam.betax;
  s->alphax = d.beam.alphax;
  s->betay = d.beam.betay;
  s->alphay = d.beam.alphay;
  s->current = d.current;
  s->nrun = d.und.nstep();
  for (int i = 0; i < d.und.nstep(); ++i)
    if (d.und.steps[i].marker & 8) {
      s->nrun = i + 1;
      break;
    }
  s->zend = d.und.steps.back().z;
  return G4B_OK;
}

int g4h_deck_run(g4h_deck* dk, g4h_result** out) {
  if (!dk || !out) {
    set_error("g4h_deck_run: null argument");
    return G4B_ERR_ARG;
  }
  try {
    Deck& d = dk->d;
    const int ns = d.nslice;
    Beam beam;
    beam.init(ns, d.nbins, d.lambda0, d.lambda0 * d.sample, d.s0, false);
    beam.gamma_ref = d.gamma0;
    std::fill(beam.current.begin(), beam.current.end(), d.current);
    if (!d.import_beam.empty()) {
      if (!read_beam_dump(d.import_beam, beam)) return G4B_ERR_ARG;
    } else {
      const size_t n = (size_t)ns * d.npart;
      std::vector<double> x(n), y(n), px(n), py(n), g(n), th(n);
      std::vector<int64_t> off(ns + 1);
      if (g4h_load_beam(&d.beam, beam.current.data(), x.data(), y.data(), px.data(), py.data(),
                        g.data(), th.data(), off.data()) != G4B_OK)
        return G4B_ERR_ARG;
      for (int s = 0; s < ns; ++s) {
        beam.beam[s].resize(off[s + 1] - off[s]);
        for (int64_t k = off[s]; k < off[s + 1]; ++k)
          beam.beam[s][k - off[s]] = Particle{g[k], th[k], x[k], y[k], px[k], py[k]};
      }
    }
    std::vector<std::unique_ptr<Field>> fields;
    std::vector<Field*> fl;
    for (auto& fi : d.fields) {
      auto f = std::make_unique<Field>();
      f->init(ns, fi.ngrid, fi.gridmax, d.lambda0, d.lambda0 * d.sample, d.s0, fi.harm);
      std::vector<double> plane(2 * (size_t)fi.ngrid * fi.ngrid);
      if (g4h_gaussian_field(fi.ngrid, fi.gridmax, f->xlambda, fi.power, fi.waist,
                             plane.data()) != G4B_OK)
        return G4B_ERR_ARG;
      const std::complex<double> ph = std::polar(1.0, fi.phase);
      for (int s = 0; s < ns; ++s)
        for (size_t k = 0; k < plane.size() / 2; ++k)
          f->field[s][k] = std::complex<double>(plane[2 * k], plane[2 * k + 1]) * ph;
      for (auto& imp : d.import_fields)
        if (imp.harm == fi.harm && !read_field_dump(imp.file, *f)) return G4B_ERR_ARG;
      f->initSolver(d.fft, d.src_filter, d.xcut, d.ycut, d.sigmoid, true, d.low_memory);
      fl.push_back(f.get());
      fields.push_back(std::move(f));
    }
    if (d.sc_nz > 0 && d.sc_rmax > 0)  // Beam::initEField (include/Beam.h:128-133)
      beam.initEField(d.sc_rmax, d.sc_ngrid, d.sc_nz, d.sc_nphi, d.lambda0, false);
    auto res = std::make_unique<g4h_result>();
    GencoreTimers t;
    const bool isTime = d.time && ns > 1;
    // files go to &setup outputdir (relative to the deck's directory), else
    // to the deck's directory; a deck given as text without either writes none
    Setup setup;
    setup.rootname = d.rootname;
    setup.outputdir = !d.outputdir.empty() ? deck_path(d.base, d.outputdir) : d.base;
    if (d.precision == G4B_MIXED) {
      run_mixed(&beam, &fl, &setup, &d.und, isTime, d.periodic, d.filter, res->diag, &t);
      res->seconds = t.beam;
    } else {
      Gencore core;
      core.run(&beam, &fl, &setup, &d.und, isTime, false, d.periodic, true, d.filter,
               res->diag, &t);
      res->seconds = t.beam + t.field + t.slip + t.diag;
    }
    res->output_file = res->diag.output_file;
    res->nslice = ns;
    res->nfield = (int)fl.size();
    res->nsteps = t.steps;
    for (Field* f : fl) {
      std::vector<double> cells(2 * (size_t)ns * f->ngrid * f->ngrid);
      for (int s = 0; s < ns; ++s)
        std::memcpy(cells.data() + 2 * (size_t)s * f->ngrid * f->ngrid, f->field[s].data(),
                    16 * (size_t)f->ngrid * f->ngrid);
      res->field_out.push_back(std::move(cells));
      res->first.push_back(f->first);
    }
    *out = res.release();
    return G4B_OK;
  } catch (const std::exception& e) {
    set_error(e.what());
    return G4B_ERR_CUDA;
  }
}

int g4h_result_output_file(g4h_result* r, char* buf, int buflen, int* needed) {
  if (!r) {
    set_error("g4h_result_output_file: null result");
    return G4B_ERR_ARG;
  }
  if (needed) *needed = (int)r->output_file.size() + 1;
  if (buf && buflen > 0) {
    const size_t n = std::min((size_t)buflen - 1, r->output_file.size());
    std::memcpy(buf, r->output_file.data(), n);
    buf[n] = 0;
  }
  return G4B_OK;
}

int g4h_result_destroy(g4h_result* r) {
  delete r;
  return G4B_OK;
}

int g4h_result_info(g4h_result* r, int* nz, int* nslice, int* nfield, int* nsteps,
                    double* seconds) {
  if (!r) {
    set_error("g4h_result_info: null result");
    return G4B_ERR_ARG;
  }
  if (nz) *nz = (int)r->diag.zout.size();
  if (nslice) *nslice = r->nslice;
  if (nfield) *nfield = r->nfield;
  if (nsteps) *nsteps = r->nsteps;
  if (seconds) *seconds = r->seconds;
  return G4B_OK;
}

int g4h_result_keys(g4h_result* r, int group, char* buf, int buflen, int* needed) {
  if (!r || group < 0 || group > r->nfield) {
    set_error("g4h_result_keys: bad group");
    return G4B_ERR_ARG;
  }
  std::string s;
  for (auto& kv : r->diag.val[2 + group]) s += kv.first + "\n";
  if (needed) *needed = (int)s.size() + 1;
  if (buf && buflen > 0) {
    const size_t n = std::min((size_t)buflen - 1, s.size());
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
  }
  return G4B_OK;
}

int g4h_result_get(g4h_result* r, int group, const char* key, double* outv, int64_t cap,
                   int64_t* len) {
  if (!r || !key) {
    set_error("g4h_result_get: null argument");
    return G4B_ERR_ARG;
  }
  const std::vector<double>* v = nullptr;
  if (group == -1 && std::strcmp(key, "z") == 0) {
    v = &r->diag.zout;
  } else if (group >= 0 && group <= r->nfield) {
    auto& m = r->diag.val[2 + group];
    auto it = m.find(key);
    if (it != m.end()) v = &it->second;
  }
  if (!v) {
    set_error(std::string("g4h_result_get: no record ") + key);
    return G4B_ERR_ARG;
  }
  if (len) *len = (int64_t)v->size();
  if (outv) std::memcpy(outv, v->data(), 8 * std::min<int64_t>(cap, (int64_t)v->size()));
  return G4B_OK;
}

int g4h_result_field(g4h_result* r, int ifield, double* cells, int* first) {
  if (!r || ifield < 0 || ifield >= r->nfield) {
    set_error("g4h_result_field: bad field index");
    return G4B_ERR_ARG;
  }
  if (cells)
    std::memcpy(cells, r->field_out[ifield].data(), 8 * r->field_out[ifield].size());
  if (first) *first = r->first[ifield];
  return G4B_OK;
}

}  // extern "C"
