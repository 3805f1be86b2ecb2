// Reader of reference-format parameter files (deal.II ParameterHandler
// syntax: "subsection" / "set key = value" / "end", '#' comments) for the
// keys declared in mf_elasticity.h:156-607, and an evaluator of the
// boundary-condition expressions (functions of x, y, z, t).
#include "problem_internal.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <sstream>

namespace lsmf {

namespace {

std::string trim(const std::string &s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) ++a;
  while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

std::vector<std::string> split(const std::string &s, char sep) {
  std::vector<std::string> out;
  std::string cur;
  for (char c : s) {
    if (c == sep) { out.push_back(trim(cur)); cur.clear(); }
    else cur += c;
  }
  out.push_back(trim(cur));
  return out;
}

// ------------------------------------------------------------ expressions
// Recursive-descent parser producing a postfix program over a value stack.
enum Op { PUSH, VAR_X, VAR_Y, VAR_Z, VAR_T, ADD, SUB, MUL, DIV, POW, NEG, FN };

struct Parser {
  const std::string &s;
  size_t i = 0;
  std::vector<Expr::Ins> &prog;
  std::string err;
  Parser(const std::string &src, std::vector<Expr::Ins> &p) : s(src), prog(p) {}
  void ws() { while (i < s.size() && std::isspace((unsigned char)s[i])) ++i; }
  bool eat(char c) {
    ws();
    if (i < s.size() && s[i] == c) { ++i; return true; }
    return false;
  }
  bool expr() {
    if (!term()) return false;
    while (true) {
      if (eat('+')) { if (!term()) return false; prog.push_back({ADD, 0, 0}); }
      else if (eat('-')) { if (!term()) return false; prog.push_back({SUB, 0, 0}); }
      else return true;
    }
  }
  bool term() {
    if (!unary()) return false;
    while (true) {
      if (eat('*')) { if (!unary()) return false; prog.push_back({MUL, 0, 0}); }
      else if (eat('/')) { if (!unary()) return false; prog.push_back({DIV, 0, 0}); }
      else return true;
    }
  }
  bool unary() {
    if (eat('-')) { if (!unary()) return false; prog.push_back({NEG, 0, 0}); return true; }
    if (eat('+')) return unary();
    return power();
  }
  bool power() {
    if (!primary()) return false;
    if (eat('^')) {
      if (!unary()) return false;  // right associative
      prog.push_back({POW, 0, 0});
    }
    return true;
  }
  bool primary() {
    ws();
    if (i >= s.size()) { err = "unexpected end of expression"; return false; }
    if (eat('(')) {
      if (!expr()) return false;
      if (!eat(')')) { err = "missing ')'"; return false; }
      return true;
    }
    if (std::isdigit((unsigned char)s[i]) || s[i] == '.') {
      const char *b = s.c_str() + i;
      char *e = nullptr;
      const double v = std::strtod(b, &e);
      if (e == b) { err = "bad number"; return false; }
      i += (size_t)(e - b);
      prog.push_back({PUSH, v, 0});
      return true;
    }
    if (std::isalpha((unsigned char)s[i]) || s[i] == '_') {
      size_t b = i;
      while (i < s.size() && (std::isalnum((unsigned char)s[i]) || s[i] == '_')) ++i;
      const std::string id = s.substr(b, i - b);
      if (id == "x") { prog.push_back({VAR_X, 0, 0}); return true; }
      if (id == "y") { prog.push_back({VAR_Y, 0, 0}); return true; }
      if (id == "z") { prog.push_back({VAR_Z, 0, 0}); return true; }
      if (id == "t") { prog.push_back({VAR_T, 0, 0}); return true; }
      if (id == "pi") { prog.push_back({PUSH, M_PI, 0}); return true; }
      static const char *fns[] = {"sin", "cos", "tan", "exp", "log", "sqrt", "abs", "tanh", "atan"};
      for (int f = 0; f < 9; ++f)
        if (id == fns[f]) {
          if (!eat('(')) { err = "expected '(' after " + id; return false; }
          if (!expr()) return false;
          if (!eat(')')) { err = "missing ')'"; return false; }
          prog.push_back({FN, 0, f});
          return true;
        }
      err = "unknown name '" + id + "'";
      return false;
    }
    err = std::string("unexpected character '") + s[i] + "'";
    return false;
  }
};

}  // namespace

bool Expr::parse(const std::string &src, std::string &err) {
  prog.clear();
  text = src;
  Parser p(src, prog);
  if (!p.expr()) { err = p.err + " in '" + src + "'"; return false; }
  p.ws();
  if (p.i != src.size()) { err = "trailing characters in '" + src + "'"; return false; }
  return true;
}

double Expr::eval(double x, double y, double z, double t) const {
  double st[64];
  int sp = 0;
  for (const Ins &in : prog) {
    switch (in.op) {
      case PUSH: st[sp++] = in.v; break;
      case VAR_X: st[sp++] = x; break;
      case VAR_Y: st[sp++] = y; break;
      case VAR_Z: st[sp++] = z; break;
      case VAR_T: st[sp++] = t; break;
      case ADD: --sp; st[sp - 1] += st[sp]; break;
      case SUB: --sp; st[sp - 1] -= st[sp]; break;
      case MUL: --sp; st[sp - 1] *= st[sp]; break;
      case DIV: --sp; st[sp - 1] /= st[sp]; break;
      case POW: --sp; st[sp - 1] = std::pow(st[sp - 1], st[sp]); break;
      case NEG: st[sp - 1] = -st[sp - 1]; break;
      case FN: {
        double &a = st[sp - 1];
        switch (in.f) {
          case 0: a = std::sin(a); break;
          case 1: a = std::cos(a); break;
          case 2: a = std::tan(a); break;
          case 3: a = std::exp(a); break;
          case 4: a = std::log(a); break;
          case 5: a = std::sqrt(a); break;
          case 6: a = std::fabs(a); break;
          case 7: a = std::tanh(a); break;
          default: a = std::atan(a); break;
        }
        break;
      }
    }
    if (sp >= 63) return NAN;
  }
  return sp == 1 ? st[0] : NAN;
}

// ----------------------------------------------------------------- .prm
namespace {

bool to_bool(const std::string &v, bool &out) {
  std::string s = v;
  std::transform(s.begin(), s.end(), s.begin(), ::tolower);
  if (s == "true" || s == "1" || s == "yes") { out = true; return true; }
  if (s == "false" || s == "0" || s == "no") { out = false; return true; }
  return false;
}

bool to_int(const std::string &v, int &out) {
  char *e = nullptr;
  const long x = std::strtol(v.c_str(), &e, 10);
  if (e == v.c_str() || trim(e).size()) return false;
  out = (int)x;
  return true;
}

bool to_double(const std::string &v, double &out) {
  char *e = nullptr;
  const double x = std::strtod(v.c_str(), &e);
  if (e == v.c_str() || trim(e).size()) return false;
  out = x;
  return true;
}

}  // namespace

lsmf_status parse_prm(const std::string &text, ProblemParams &P) {
  std::istringstream in(text);
  std::string line;
  std::vector<std::string> stack;
  int lineno = 0;
  auto fail = [&](const std::string &msg) {
    set_error("line " + std::to_string(lineno) + ": " + msg);
    return LSMF_ERR_PRM;
  };
  while (std::getline(in, line)) {
    ++lineno;
    const size_t hash = line.find('#');
    if (hash != std::string::npos) line = line.substr(0, hash);
    line = trim(line);
    if (line.empty()) continue;
    if (line.rfind("subsection", 0) == 0) {
      stack.push_back(trim(line.substr(10)));
      continue;
    }
    if (line == "end") {
      if (stack.empty()) return fail("'end' without subsection");
      stack.pop_back();
      continue;
    }
    if (line.rfind("set", 0) != 0) return fail("expected 'set', 'subsection' or 'end'");
    const size_t eq = line.find('=');
    if (eq == std::string::npos) return fail("missing '='");
    const std::string key = trim(line.substr(3, eq - 3)), val = trim(line.substr(eq + 1));
    const std::string sec = stack.empty() ? "" : stack.back();
    bool ok = true, known = true;
    if (sec == "Finite element system") {
      if (key == "Polynomial degree") ok = to_int(val, P.degree);
      else if (key == "Quadrature order") ok = to_int(val, P.quad_order);
      else known = false;
    } else if (sec == "Geometry") {
      if (key == "Elements per edge") ok = to_int(val, P.elements_per_edge);
      else if (key == "Global refinement") ok = to_int(val, P.n_refinements);
      else if (key == "Grid scale") ok = to_double(val, P.scale);
      else if (key == "Extrusion height") ok = to_double(val, P.extrusion_height);
      else if (key == "Extrusion slices") ok = to_int(val, P.extrusion_slices);
      else if (key == "Dimension") ok = to_int(val, P.dim);
      else if (key == "Type") P.type = val;
      else if (key == "Box cells") {  // additive: coarse cells "nx, ny, nz"
        auto v = split(val, ',');
        ok = v.size() == 3 && to_int(v[0], P.box_cells[0]) && to_int(v[1], P.box_cells[1]) && to_int(v[2], P.box_cells[2]);
      } else if (key == "Box lower corner" || key == "Box upper corner") {
        auto v = split(val, ',');
        double *dst = key == "Box lower corner" ? P.box_lo : P.box_hi;
        ok = v.size() == 3 && to_double(v[0], dst[0]) && to_double(v[1], dst[1]) && to_double(v[2], dst[2]);
      } else if (key == "Cook thickness") ok = to_double(val, P.cook_thickness);
      else if (key == "Void spheres") {  // additive: "count, radius, seed"
        auto v = split(val, ',');
        ok = v.size() == 3 && to_int(v[0], P.void_count) && to_double(v[1], P.void_radius) && to_int(v[2], P.void_seed);
      } else known = false;
    } else if (sec == "Material properties") {
      if (key == "Poisson's ratio") ok = to_double(val, P.nu);
      else if (key == "Shear modulus") ok = to_double(val, P.mu);
      else if (key == "Formulation") ok = to_int(val, P.formulation);
      else known = false;
    } else if (sec == "Linear solver") {
      if (key == "Solver type") P.solver_type = val;
      else if (key == "Residual") ok = to_double(val, P.tol_lin);
      else if (key == "Max iteration multiplier") ok = to_int(val, P.max_it_mult);
      else if (key == "Preconditioner type") P.precond = val;
      else if (key == "Preconditioner relaxation") ok = to_double(val, P.relaxation);
      else if (key == "Preconditioner AMG aggregation threshold") ok = to_double(val, P.amg_threshold);
      else if (key == "Condition number CG iterations") ok = to_int(val, P.cond_cg_its);
      else if (key == "MF caching") P.caching = val;
      else if (key == "MF Chebyshev number CG iterations") ok = to_int(val, P.cheb_eig_its);
      else if (key == "MF Chebyshev coarse") ok = to_bool(val, P.coarse_chebyshev);
      else if (key == "MF Chebyshev coarse accurate eigenvalues") ok = to_bool(val, P.coarse_accurate_eig);
      else if (key == "MF level precision") P.level_precision = val;             // additive
      else if (key == "MF Chebyshev degree") ok = to_int(val, P.cheb_degree);     // additive
      else if (key == "MF Chebyshev smoothing range") ok = to_double(val, P.smoothing_range);  // additive
      else if (key == "MF scatter") P.scatter = val;                             // additive
      else known = false;
    } else if (sec == "Nonlinear solver") {
      if (key == "Max iterations Newton-Raphson") ok = to_int(val, P.max_nr);
      else if (key == "Tolerance force") ok = to_double(val, P.tol_f);
      else if (key == "Absolute tolerance force") ok = to_double(val, P.tol_f_abs);
      else if (key == "Tolerance displacement") ok = to_double(val, P.tol_u);
      else if (key == "Absolute tolerance displacement") ok = to_double(val, P.tol_u_abs);
      else known = false;
    } else if (sec == "Time") {
      if (key == "End time") ok = to_double(val, P.end_time);
      else if (key == "Time step size") ok = to_double(val, P.dt);
      else known = false;
    } else if (sec == "Misc") {
      if (key == "Output folder") P.output_folder = val;
      else if (key == "Output solution") ok = to_bool(val, P.output_solution);
      else if (key == "Always assemble tangent") ok = to_bool(val, P.always_assemble);
      else if (key == "Output absolute norms") ok = to_bool(val, P.output_abs_norms);
      else if (key == "Output points") {
        P.output_points.clear();
        if (!val.empty())
          for (const std::string &pt : split(val, ';')) {
            auto v = split(pt, ',');
            std::array<double, 3> p{0, 0, 0};
            if (v.size() < 2 || v.size() > 3) { ok = false; break; }
            for (size_t k = 0; k < v.size(); ++k) ok = ok && to_double(v[k], p[k]);
            P.output_points.push_back(p);
          }
      } else known = false;
    } else if (sec == "Boundary conditions") {
      if (key == "Dirichlet IDs and expressions" || key == "Neumann IDs and expressions") {
        std::vector<BCExpr> &dst = key[0] == 'D' ? P.dirichlet : P.neumann;
        dst.clear();
        if (!val.empty())
          for (const std::string &ent : split(val, ';')) {
            const size_t c = ent.find(':');
            if (c == std::string::npos) { ok = false; break; }
            BCExpr b;
            if (!to_int(trim(ent.substr(0, c)), b.id)) { ok = false; break; }
            auto comps = split(ent.substr(c + 1), ',');
            if (comps.size() != 3) return fail("expected 3 components for boundary id " + std::to_string(b.id));
            for (int k = 0; k < 3; ++k) {
              std::string e;
              if (!b.expr[k].parse(comps[k], e)) return fail(e);
            }
            dst.push_back(b);
          }
      } else if (key == "Dirichlet IDs and component mask") {
        P.dirichlet_mask.clear();
        if (!val.empty())
          for (const std::string &ent : split(val, ';')) {
            const size_t c = ent.find(':');
            int id = 0;
            if (c == std::string::npos || !to_int(trim(ent.substr(0, c)), id)) { ok = false; break; }
            auto comps = split(ent.substr(c + 1), ',');
            if (comps.size() != 3) { ok = false; break; }
            int mask = 0;
            for (int k = 0; k < 3; ++k) {
              bool b;
              if (!to_bool(comps[k], b)) { ok = false; break; }
              if (b) mask |= 1 << k;
            }
            P.dirichlet_mask[id] = mask;
          }
      } else known = false;
    } else {
      known = false;
    }
    if (!known) return fail("undeclared entry '" + key + "' in subsection '" + sec + "'");
    if (!ok) return fail("invalid value '" + val + "' for '" + key + "'");
  }
  if (!stack.empty()) return fail("missing 'end' for subsection '" + stack.back() + "'");
  return LSMF_OK;
}

}  // namespace lsmf
