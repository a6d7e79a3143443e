// g4h_lattice.cpp -- .lat parsing and expansion into per-step tables.
//
// The reference reads lattices through upstream GENESIS 1.3 v4 (Lattice,
// LatticeElements, Undulator; not in the reference tree).  This file parses
// the subset used by the reference's test deck (test/fel.lat:1-11) and the
// benchmark lattices, and fills the per-step values the hot path consumes.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "Undulator.h"
#include "g4h.h"
#include "g4h_internal.h"

namespace g4h {

double coupling(double aw, int harm, bool helical) {
  if (harm < 1) return 0.0;
  if (helical) return harm == 1 ? aw : 0.0;
  if (harm % 2 == 0) return 0.0;  // planar: no on-axis coupling at even h
  const double xi = harm * aw * aw / (2.0 * (1.0 + aw * aw));
  const int m = (harm - 1) / 2;
  const double jj = std::cyl_bessel_j((double)m, xi) - std::cyl_bessel_j((double)m + 1, xi);
  return aw * ((m % 2) ? -jj : jj);
}

double Undulator::fc(int harm) const { return fc_at(istep_, harm); }

double Undulator::fc_at(int i, int harm) const {
  const LatticeStep& s = steps[i];
  if (!s.st.in_undulator) return 0.0;
  return coupling(s.st.aw, harm, s.helical != 0);
}

namespace {

struct Element {
  std::string type;  // upper case
  std::map<std::string, std::string> par;
  std::vector<std::pair<int, std::string>> line;  // for LINE
};

std::string upper(std::string s) {
  for (auto& c : s) c = (char)std::toupper((unsigned char)c);
  return s;
}

std::string trim(const std::string& s) {
  size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
  return a == std::string::npos ? "" : s.substr(a, b - a + 1);
}

double num(const Element& e, const char* key, double def) {
  auto it = e.par.find(key);
  if (it == e.par.end()) return def;
  const std::string v = upper(it->second);
  if (v == "TRUE" || v == "T") return 1.0;
  if (v == "FALSE" || v == "F") return 0.0;
  return std::atof(it->second.c_str());
}

bool parse(const std::string& text0, std::map<std::string, Element>& out) {
  std::string text;
  {  // strip comments
    std::istringstream is(text0);
    std::string ln;
    while (std::getline(is, ln)) {
      auto h = ln.find('#');
      if (h != std::string::npos) ln = ln.substr(0, h);
      text += ln + "\n";
    }
  }
  size_t pos = 0;
  while (true) {
    const size_t semi = text.find(';', pos);
    const std::string stmt = trim(text.substr(pos, semi == std::string::npos ? std::string::npos : semi - pos));
    if (!stmt.empty()) {
      const size_t colon = stmt.find(':');
      const size_t eq = stmt.find('=', colon == std::string::npos ? 0 : colon);
      const size_t lb = stmt.find('{'), rb = stmt.rfind('}');
      if (colon == std::string::npos || eq == std::string::npos || lb == std::string::npos ||
          rb == std::string::npos) {
        set_error("lattice: cannot parse statement '" + stmt + "'");
        return false;
      }
      Element e;
      const std::string label = upper(trim(stmt.substr(0, colon)));
      e.type = upper(trim(stmt.substr(colon + 1, eq - colon - 1)));
      const std::string body = stmt.substr(lb + 1, rb - lb - 1);
      std::istringstream bs(body);
      std::string item;
      while (std::getline(bs, item, ',')) {
        item = trim(item);
        if (item.empty()) continue;
        if (e.type == "LINE") {
          int rep = 1;
          const size_t star = item.find('*');
          std::string name = item;
          if (star != std::string::npos) {
            rep = std::atoi(item.substr(0, star).c_str());
            name = trim(item.substr(star + 1));
          }
          e.line.push_back({rep, upper(name)});
        } else {
          const size_t q = item.find('=');
          if (q == std::string::npos) {
            set_error("lattice: bad parameter '" + item + "' in " + label);
            return false;
          }
          std::string key = trim(item.substr(0, q));
          for (auto& c : key) c = (char)std::tolower((unsigned char)c);
          e.par[key] = trim(item.substr(q + 1));
        }
      }
      out[label] = e;
    }
    if (semi == std::string::npos) break;
    pos = semi + 1;
  }
  return true;
}

bool expand(const std::map<std::string, Element>& el, const std::string& name,
            std::vector<const Element*>& flat, int depth) {
  if (depth > 64) {
    set_error("lattice: line nesting too deep (recursive LINE?)");
    return false;
  }
  auto it = el.find(name);
  if (it == el.end()) {
    set_error("lattice: unknown element or line '" + name + "'");
    return false;
  }
  if (it->second.type != "LINE") {
    flat.push_back(&it->second);
    return true;
  }
  for (auto& [rep, sub] : it->second.line)
    for (int r = 0; r < rep; ++r)
      if (!expand(el, sub, flat, depth + 1)) return false;
  return true;
}

double chicane_angle(double delay, double lb, double ld) {
  if (delay <= 0 || lb <= 0) return 0.0;
  auto f = [&](double t) {
    return 4 * lb * (t / std::sin(t) - 1) + 2 * ld * (1 / std::cos(t) - 1) - delay;
  };
  double lo = 1e-12, hi = 1.5;
  if (f(hi) < 0) return hi;
  for (int i = 0; i < 200; ++i) {
    const double mid = 0.5 * (lo + hi);
    (f(mid) > 0 ? hi : lo) = mid;
  }
  return 0.5 * (lo + hi);
}

}  // namespace

bool build_lattice(const std::string& text, const std::string& beamline, double delz,
                   double gamma0, double lambda0, Undulator& und) {
  if (!(delz > 0) || !(gamma0 > 1) || !(lambda0 > 0)) {
    set_error("lattice: delz, gamma0 and lambda0 must be positive");
    return false;
  }
  std::map<std::string, Element> el;
  if (!parse(text, el)) return false;
  std::vector<const Element*> flat;
  if (!expand(el, upper(beamline), flat, 0)) return false;
  und.steps.clear();
  und.gamma0 = gamma0;
  und.lambda0 = lambda0;
  double z = 0.0;
  const double g2 = 2.0 * gamma0 * gamma0;
  auto blank = [&]() {
    LatticeStep s;
    s.st.gamma_ref = gamma0;
    return s;
  };
  for (const Element* e : flat) {
    const std::string& t = e->type;
    if (t == "MARKER") {
      int m = 0;
      if (num(*e, "dumpbeam", 0) != 0) m |= 1;
      if (num(*e, "dumpfield", 0) != 0) m |= 2;
      if (num(*e, "sort", 0) != 0) m |= 4;
      if (num(*e, "stop", 0) != 0) m |= 8;
      if (!und.steps.empty()) und.steps.back().marker |= m;
      continue;
    }
    if (t == "UNDULATOR") {
      const double lu = num(*e, "lambdau", 0), nw = num(*e, "nwig", 0);
      const double aw = num(*e, "aw", 0);
      const bool hel = num(*e, "helical", 0) != 0;
      const double ku = lu > 0 ? 2 * M_PI / lu : 0;
      const double kx = num(*e, "kx", hel ? 0.5 : 0.0), ky = num(*e, "ky", hel ? 0.5 : 1.0);
      const double taper = num(*e, "taper", 0.0);  // linear d(aw)/aw over the element
      const double L = lu * nw;
      const int ns = std::max(1, (int)std::lround(L / delz));
      for (int i = 0; i < ns; ++i) {
        LatticeStep s = blank();
        const double dz = L / ns;
        const double awi = aw * (1.0 + taper * (i + 0.5) / ns);
        s.st.delz = dz;
        s.st.aw = awi;
        s.st.ku = ku;
        s.st.kx = kx * ku * ku;
        s.st.ky = ky * ku * ku;
        s.st.ax = num(*e, "ax", 0);
        s.st.ay = num(*e, "ay", 0);
        s.st.gradx = num(*e, "gradx", 0);
        s.st.grady = num(*e, "grady", 0);
        s.st.in_undulator = awi > 0 ? 1 : 0;
        s.helical = hel;
        s.slip = dz * (1 + awi * awi) / g2 / lambda0;
        z += dz;
        s.z = z;
        und.steps.push_back(s);
      }
      continue;
    }
    const double L = num(*e, "l", 0.0);
    if (t == "CHICANE") {
      LatticeStep s = blank();
      const double lb = num(*e, "lb", 0), ld = num(*e, "ld", 0), delay = num(*e, "delay", 0);
      s.st.delz = L;
      s.st.chic_angle = chicane_angle(delay, lb, ld);
      s.st.chic_lb = lb;
      s.st.chic_ld = ld;
      s.st.chic_lt = L;
      s.slip = L / g2 / lambda0 + delay / lambda0;
      z += L;
      s.z = z;
      und.steps.push_back(s);
      continue;
    }
    if (t != "DRIFT" && t != "QUADRUPOLE" && t != "CORRECTOR" && t != "PHASESHIFTER") {
      set_error("lattice: unsupported element type " + t);
      return false;
    }
    if (L <= 0) {
      if (t == "CORRECTOR" && !und.steps.empty()) {
        und.steps.back().st.cx += num(*e, "cx", 0);
        und.steps.back().st.cy += num(*e, "cy", 0);
      }
      if (t == "PHASESHIFTER" && !und.steps.empty())
        und.steps.back().st.autophase += num(*e, "phi", 0);
      continue;
    }
    const int ns = std::max(1, (int)std::ceil(L / delz - 1e-9));
    for (int i = 0; i < ns; ++i) {
      LatticeStep s = blank();
      const double dz = L / ns;
      s.st.delz = dz;
      if (t == "QUADRUPOLE") {
        s.st.qf = num(*e, "k1", 0);
        s.st.dqx = num(*e, "dx", 0);
        s.st.dqy = num(*e, "dy", 0);
      }
      if (t == "CORRECTOR" && i == ns - 1) {
        s.st.cx = num(*e, "cx", 0);
        s.st.cy = num(*e, "cy", 0);
      }
      if (t == "PHASESHIFTER" && i == 0) s.st.autophase = num(*e, "phi", 0);
      s.slip = dz / g2 / lambda0;
      z += dz;
      s.z = z;
      und.steps.push_back(s);
    }
  }
  if (und.steps.empty()) {
    set_error("lattice: beamline has no steps");
    return false;
  }
  und.reset();
  return true;
}

}  // namespace g4h

struct g4h_lattice {
  g4h::Undulator und;
};

using namespace g4h;

extern "C" {

double g4h_coupling(double aw, int harm, int helical) { return coupling(aw, harm, helical != 0); }

int g4h_lattice_parse(const char* text, const char* beamline, double delz, double gamma0,
                      double lambda0, g4h_lattice** out) {
  if (!text || !beamline || !out) {
    set_error("g4h_lattice_parse: null argument");
    return G4B_ERR_ARG;
  }
  auto lat = std::make_unique<g4h_lattice>();
  if (!build_lattice(text, beamline, delz, gamma0, lambda0, lat->und)) return G4B_ERR_ARG;
  *out = lat.release();
  return G4B_OK;
}

int g4h_lattice_destroy(g4h_lattice* lat) {
  delete lat;
  return G4B_OK;
}

int g4h_lattice_nstep(g4h_lattice* lat, int* n) {
  if (!lat || !n) {
    set_error("g4h_lattice_nstep: null argument");
    return G4B_ERR_ARG;
  }
  *n = lat->und.nstep();
  return G4B_OK;
}

int g4h_lattice_step(g4h_lattice* lat, int i, g4b_step* st, double* slip, double* z,
                     int* marker) {
  if (!lat || i < 0 || i >= lat->und.nstep()) {
    set_error("g4h_lattice_step: bad argument");
    return G4B_ERR_ARG;
  }
  const LatticeStep& s = lat->und.steps[i];
  if (st) *st = s.st;
  if (slip) *slip = s.slip;
  if (z) *z = s.z;
  if (marker) *marker = s.marker;
  return G4B_OK;
}

int g4h_lattice_fc(g4h_lattice* lat, int i, int harm, double* fc) {
  if (!lat || !fc || i < 0 || i >= lat->und.nstep()) {
    set_error("g4h_lattice_fc: bad argument");
    return G4B_ERR_ARG;
  }
  *fc = lat->und.fc_at(i, harm);
  return G4B_OK;
}

}  // extern "C"
