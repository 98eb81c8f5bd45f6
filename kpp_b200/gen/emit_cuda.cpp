// kppcu CUDA emitter.
//
// Writes one header, <prefix>.cuh, holding the mechanism as sm_100a device
// code plus the host-side tables the C-ABI exports:
//   kpp_update_rconst  rate constants (the mechanism's rate expressions,
//                      src/gen.c:2343-2473, with the rate-law functions of
//                      util/UserRateLaws.c as device functions)
//   kpp_fun            ODE right-hand side, aggregate form (src/gen.c:642-724)
//   kpp_jac_sp         sparse Jacobian in the LU pattern (src/gen.c:1185-1322)
//   kpp_decomp         fully unrolled no-pivot sparse LU; same operation
//                      sequence as the loop of util/sutil.c:2-23
//   kpp_solve          unrolled forward/backward substitution
//                      (src/gen.c:1960-2034)
// and a second header, <prefix>_cmplx.cuh, with the complex LU the
// Runge-Kutta methods factorise (KppDecompCmplxR / KppSolveCmplxR of
// util/sutil.c:28-90: unrolled in the same operation order, or for patterns
// of 2000 entries or more the generic loops over the LU tables, as are the
// real LU and solve of such mechanisms).
//
// Arithmetic is the reference's, operation for operation: expression trees
// are built with the same constant folding (multiplying by a constant 1
// drops the constant, a constant 0 annihilates, adding 0 drops the term,
// src/code.c:519-590), constants are the single-precision values KPP stores,
// written with "%g" (src/code.c:474-476, src/code_c.c:66), sums run left to
// right over equations in order, and the printed expressions are
// parenthesised so that C evaluates exactly the tree.  Built without FMA
// contraction the device code then rounds like the reference's C code; only
// the libm-class functions (exp, pow, log10, cos) can differ by an ulp.
#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <fstream>
#include <memory>
#include <set>
#include <sstream>
#include <vector>

#include "mechanism.hpp"

namespace kppcu {

namespace {

// ---------------------------------------------------------------------------
// Expression trees
// ---------------------------------------------------------------------------
enum NodeKind { N_CONST, N_LEAF, N_ADD, N_SUB, N_MUL, N_DIV };

struct Node;
using P = std::shared_ptr<Node>;

struct Node {
  NodeKind kind;
  int sign = 1;      // leaves and constants carry a sign
  float value = 0;   // |constant|, single precision
  std::string text;  // leaf text
  P l, r;
};

P cnst(double v) {
  P n = std::make_shared<Node>();
  n->kind = N_CONST;
  float f = (float)v;
  if (f < 0) { f = -f; n->sign = -1; }
  n->value = f;
  return n;
}
P leaf(const std::string& t) {
  P n = std::make_shared<Node>();
  n->kind = N_LEAF;
  n->text = t;
  return n;
}
P bin(NodeKind k, P a, P b) {
  P n = std::make_shared<Node>();
  n->kind = k;
  n->l = std::move(a);
  n->r = std::move(b);
  return n;
}
bool is_const(const P& n, float v) { return n && n->kind == N_CONST && n->value == v; }

P add(P a, P b) {
  if (!a) return b;
  if (!b) return a;
  if (is_const(a, 0)) return b;
  if (is_const(b, 0)) return a;
  return bin(N_ADD, a, b);
}
P sub(P a, P b) {
  if (!a) return bin(N_SUB, nullptr, b);
  if (!b) return a;
  if (is_const(a, 0)) return bin(N_SUB, nullptr, b);
  if (is_const(b, 0)) return a;
  return bin(N_SUB, a, b);
}
P mul(P a, P b) {
  if (!a) return b;
  if (!b) return a;
  if (is_const(a, 1)) { b->sign *= a->sign; return b; }
  if (is_const(b, 1)) return a;  // the sign of b is not applied (src/code.c:555-559)
  if (is_const(a, 0)) return a;
  if (is_const(b, 0)) return b;
  return bin(N_MUL, a, b);
}
P divide(P a, P b) {
  if (!a) return bin(N_DIV, cnst(1), b);
  if (!b) return a;
  if (is_const(b, 1)) return a;
  return bin(N_DIV, a, b);
}

std::string fmt_g(float v) {
  char buf[64];
  std::snprintf(buf, sizeof buf, "%g", (double)v);
  std::string s = buf;
  // make it a double literal without changing its value
  if (s.find_first_of(".eEn") == std::string::npos) s += ".0";
  return s;
}

int prec(const P& n) {
  switch (n->kind) {
    case N_ADD: case N_SUB: return 1;
    case N_MUL: case N_DIV: return 2;
    default: return 3;
  }
}

// C text that evaluates exactly the tree: left-associative chains print
// without parentheses, anything else is parenthesised.
std::string print(const P& n, int parent, bool right) {
  std::string s;
  switch (n->kind) {
    case N_CONST: s = fmt_g(n->value); return n->sign < 0 ? "(-" + s + ")" : s;
    case N_LEAF: return n->sign < 0 ? "(-" + n->text + ")" : n->text;
    case N_ADD: s = print(n->l, 1, false) + " + " + print(n->r, 1, true); break;
    case N_SUB:
      s = n->l ? print(n->l, 1, false) + " - " + print(n->r, 1, true) : "-" + print(n->r, 3, true);
      break;
    case N_MUL: s = print(n->l, 2, false) + "*" + print(n->r, 2, true); break;
    case N_DIV: s = print(n->l, 2, false) + "/" + print(n->r, 2, true); break;
  }
  int p = prec(n);
  if (p < parent || (right && p == parent)) return "(" + s + ")";
  return s;
}
std::string print(const P& n) { return print(n, 0, false); }

// FP64 add/sub/mul/div operations the tree evaluates (unary minus is free).
long count_ops(const P& n) {
  if (!n) return 0;
  switch (n->kind) {
    case N_ADD: case N_MUL: case N_DIV: return 1 + count_ops(n->l) + count_ops(n->r);
    case N_SUB: return (n->l ? 1 : 0) + count_ops(n->l) + count_ops(n->r);
    default: return 0;
  }
}

// ---------------------------------------------------------------------------
// Mechanism accessors in the final species order
// ---------------------------------------------------------------------------
struct View {
  const Mechanism& m;
  explicit View(const Mechanism& mm) : m(mm) {}
  float left(int spc, int eq) const { return m.left[m.spc_slot[spc]][eq]; }
  float net(int spc, int eq) const { return m.net[m.spc_slot[spc]][eq]; }
  std::string name(int spc) const { return m.table[m.order[m.spc_slot[spc]]].name; }
  // rate factor: RCT[j] for expressions, the float constant for numbers
  P rconst(int eq) const {
    const Reaction& r = m.reactions[eq];
    if (r.kind == RATE_NUMBER) return cnst(r.number);
    return leaf("RCT[" + std::to_string(eq) + "]");
  }
  // product of the reactant concentrations of equation eq, leaving out one
  // occurrence of variable species `skip` (-1: none)
  P reactants(P prod, int eq, int skip) const {
    for (int i = 0; i < m.nvar; i++) {
      int k = (int)left(i, eq) - (i == skip ? 1 : 0);
      for (int c = 0; c < k; c++) prod = mul(prod, leaf("V[" + std::to_string(i) + "]"));
    }
    for (int i = m.nvar; i < m.nspec; i++) {
      int k = (int)left(i, eq);
      for (int c = 0; c < k; c++) prod = mul(prod, leaf("F[" + std::to_string(i - m.nvar) + "]"));
    }
    return prod;
  }
};

std::string c_string(const std::string& s) {
  std::string o = "\"";
  for (char c : s) {
    if (c == '"' || c == '\\') o += '\\';
    o += c;
  }
  return o + "\"";
}

void emit_int_table(std::ostream& o, const char* name, const std::vector<int>& v) {
  o << "static const int " << name << "[" << (v.empty() ? 1 : v.size()) << "] = {";
  for (size_t i = 0; i < v.size(); i++) o << (i % 16 == 0 ? "\n    " : " ") << v[i] << ",";
  if (v.empty()) o << "0";
  o << "};\n";
}

enum RateClass { RC_STATIC = 0, RC_SUN = 1, RC_DYNAMIC = 2 };

// Names declared by `double ...;` statements of an inline block (the
// variables it makes available to the rate expressions).
std::set<std::string> declared_names(const std::string& code) {
  std::set<std::string> out;
  size_t p = 0;
  while ((p = code.find("double", p)) != std::string::npos) {
    bool word_start = p == 0 || !(std::isalnum((unsigned char)code[p - 1]) || code[p - 1] == '_');
    size_t q = p + 6;
    p = q;
    if (!word_start || q >= code.size() || !std::isspace((unsigned char)code[q])) continue;
    size_t end = code.find(';', q);
    if (end == std::string::npos) break;
    std::string decl = code.substr(q, end - q);
    int depth = 0;
    bool want = true;
    for (size_t i = 0; i < decl.size(); i++) {
      char c = decl[i];
      if (c == '(' || c == '[') depth++;
      else if (c == ')' || c == ']') depth--;
      else if (c == ',' && depth == 0) want = true;
      else if (c == '=' && depth == 0) want = false;
      else if (want && (std::isalpha((unsigned char)c) || c == '_')) {
        size_t b = i;
        while (i < decl.size() && (std::isalnum((unsigned char)decl[i]) || decl[i] == '_')) i++;
        out.insert(decl.substr(b, i - b));
        want = false;
        i--;
      }
    }
    p = end;
  }
  return out;
}

// What a rate expression depends on: only TEMP/CFACTOR and pure functions
// (static for a cell), also SUN, or anything else (time, concentrations,
// user variables: recomputed at every evaluation).
int classify_rate(const std::string& e, const std::set<std::string>& static_names = {},
                  const std::set<std::string>& sun_names = {}) {
  static const char* pure[] = {"ARR_abc", "ARR_ab", "ARR_ac", "EP2", "EP3", "FALL", "exp",
                               "pow", "log", "log10", "sqrt", "cos", "sin", "tan", "fabs",
                               "fmin", "fmax", "expf", "powf", "logf", "log10f", "sqrtf",
                               "cosf", "sinf", "tanf", "fabsf", "fminf", "fmaxf", "TEMP",
                               "CFACTOR", "double", "float"};
  int cls = RC_STATIC;
  size_t i = 0;
  while (i < e.size()) {
    char c = e[i];
    if (std::isdigit((unsigned char)c) || (c == '.' && i + 1 < e.size() && std::isdigit((unsigned char)e[i + 1]))) {
      while (i < e.size() && (std::isdigit((unsigned char)e[i]) || e[i] == '.')) i++;
      if (i < e.size() && std::strchr("eEdD", e[i])) {
        size_t k = i + 1;
        if (k < e.size() && (e[k] == '+' || e[k] == '-')) k++;
        if (k < e.size() && std::isdigit((unsigned char)e[k])) {
          i = k;
          while (i < e.size() && std::isdigit((unsigned char)e[i])) i++;
        }
      }
      if (i < e.size() && std::strchr("fFlL", e[i])) i++;  // C literal suffix
      continue;
    }
    if (std::isalpha((unsigned char)c) || c == '_') {
      size_t b = i;
      while (i < e.size() && (std::isalnum((unsigned char)e[i]) || e[i] == '_')) i++;
      std::string id = e.substr(b, i - b);
      bool known = false;
      for (const char* p : pure)
        if (id == p) known = true;
      if (known || static_names.count(id)) continue;
      if (id == "SUN" || sun_names.count(id)) cls = std::max(cls, (int)RC_SUN);
      else cls = RC_DYNAMIC;
      continue;
    }
    i++;
  }
  return cls;
}


// The double value C gives to the constant kppcu prints for float v.
double const_value(float v) { return std::strtod(fmt_g(v).c_str(), nullptr); }

// Head of a product tree built by mul(rate, stoich) in the reference's
// folding: returns (rate index or -1, k1, k2) with value = (rate index >= 0 ?
// RCT[idx] : k1) * (k2 unless k2 == 1).  Multiplying by an exact 1.0 changes
// nothing, so applying k2 = 1 would also be exact; it is skipped.
struct Head {
  int rct;
  double k1, k2;
};

Head head_of(const Mechanism& m, int eq, float stoich /* 1 for Fun */) {
  const Reaction& r = m.reactions[eq];
  Head h{-1, 1.0, 1.0};
  if (r.kind != RATE_NUMBER) {
    h.rct = eq;
    h.k2 = (stoich == 1.0f) ? 1.0 : const_value(stoich);
    return h;
  }
  float c = r.number;
  if (stoich == 1.0f) { h.k1 = const_value(c); return h; }
  if (c == 1.0f) { h.k1 = const_value(stoich); return h; }
  h.k1 = const_value(c);
  h.k2 = const_value(stoich);
  return h;
}

template <class T>
void emit_table(std::ostream& o, const char* type, const char* name, const std::vector<T>& v) {
  o << "__device__ const " << type << " " << name << "[" << (v.empty() ? 1 : v.size()) << "] = {";
  for (size_t i = 0; i < v.size(); i++) o << (i % 12 == 0 ? "\n    " : " ") << v[i] << ",";
  if (v.empty()) o << "0";
  o << "};\n";
}

void emit_dtable(std::ostream& o, const char* name, const std::vector<double>& v) {
  o << "__device__ const double " << name << "[" << (v.empty() ? 1 : v.size()) << "] = {";
  for (size_t i = 0; i < v.size(); i++) {
    char buf[40];
    std::snprintf(buf, sizeof buf, "%.17g", v[i]);
    o << (i % 6 == 0 ? "\n    " : " ") << buf << ",";
  }
  if (v.empty()) o << "0";
  o << "};\n";
}

// ---------------------------------------------------------------------------
// Tables of the warp-per-cell kernel (csrc/kpp_coop.cuh)
// ---------------------------------------------------------------------------
// One warp integrates one cell whose work set sits in shared memory; its 32
// lanes share every phase through static schedules computed here.  Every value
// is produced by exactly the operation sequence of the unrolled functions
// above; only operations that do not depend on each other run side by side:
//   products  the equation rates A (Fun) and the partial derivatives B (Jac):
//             product t on lane t % 32 in round t / 32, as the weight (rate
//             constant times stoichiometric factor, the reference's leading
//             factors) times the reactant concentrations in order
//   sums      each Vdot row / Jacobian entry summed by one lane in equation
//             order; outputs spread over lanes, longest sums first
//   LU        the operations of util/sutil.c's loop (row entry divided by the
//             pivot; pivot row times the multiplier subtracted) as a dependency
//             graph, list-scheduled by longest remaining path into iterations
//             separated by warp barriers, each iteration of one kind
//   forward   substitution: a lane owns a row's left-to-right sum and runs
//             its terms as soon as their operands are final (written by
//             another lane in an earlier iteration); the backward substitution
//             runs on one lane as the unrolled kpp_solve_bw
// All tables are 32-bit words in one array that each CTA stages in shared
// memory.  A phase that iterates holds, per iteration, how many entries each
// lane runs (4-bit counts, eight lanes per word) and, per lane, its entries in
// order (layout [position][lane], so the lanes of a warp read consecutive
// words).
// LU patterns of this many entries or more get the loop forms of KppDecomp,
// KppSolve and the complex LU instead of unrolled code.
constexpr int kGenericLu = 2000;

constexpr int kCoopLanes = 32;
constexpr int kCoopLuCap = 2;     // LU units per lane per iteration
constexpr int kCoopSolveCap = 4;  // solve terms per lane per iteration

int bits_for(long n) {
  int b = 1;
  while ((1L << b) < n) b++;
  return b;
}

struct CoopStream {
  std::vector<std::vector<unsigned>> lane = std::vector<std::vector<unsigned>>(kCoopLanes);
  std::vector<std::vector<int>> count;  // [iteration][lane]
  size_t max_len() const {
    size_t n = 0;
    for (auto& l : lane) n = std::max(n, l.size());
    return n;
  }
  // entries as [position][lane], padded with `pad`
  std::vector<unsigned> interleaved(unsigned pad) const {
    const size_t len = max_len();
    std::vector<unsigned> out(len * kCoopLanes, pad);
    for (int l = 0; l < kCoopLanes; l++)
      for (size_t k = 0; k < lane[l].size(); k++) out[k * kCoopLanes + l] = lane[l][k];
    return out;
  }
  // per-iteration counts, eight 4-bit lanes per word
  std::vector<unsigned> counts() const {
    std::vector<unsigned> out;
    for (auto& c : count)
      for (int w = 0; w < kCoopLanes / 8; w++) {
        unsigned word = 0;
        for (int j = 0; j < 8; j++) word |= (unsigned)c[w * 8 + j] << (4 * j);
        out.push_back(word);
      }
    return out;
  }
};

// LU: units in the order of util/sutil.c's loop; entry = div<<31 | t<<2B | m<<B | s
// (div: J[t] = J[t] / J[s]; else J[t] = J[t] + (-J[m]) * J[s]).
CoopStream coop_schedule_lu(const Mechanism& m, int B) {
  const int n = m.nvar;
  std::vector<std::vector<int>> pos(n, std::vector<int>(n, -1));
  for (int k = 0; k < m.lu_nonzero; k++) pos[m.lu_irow[k]][m.lu_icol[k]] = k;
  struct Unit { int div, t, mm, s; };
  std::vector<Unit> u;
  std::vector<std::vector<int>> deps;
  std::vector<int> last(m.lu_nonzero, -1);
  auto dep = [&](std::vector<int>& d, int e) {
    if (last[e] >= 0) d.push_back(last[e]);
  };
  for (int k = 0; k < n; k++)
    for (int kk = m.lu_crow[k]; kk < m.lu_diag[k]; kk++) {
      const int j = m.lu_icol[kk];
      std::vector<int> d;
      dep(d, kk);
      dep(d, m.lu_diag[j]);
      u.push_back({1, kk, 0, m.lu_diag[j]});
      deps.push_back(d);
      last[kk] = (int)u.size() - 1;
      for (int jj = m.lu_diag[j] + 1; jj < m.lu_crow[j + 1]; jj++) {
        const int t = pos[k][m.lu_icol[jj]];
        std::vector<int> d2;
        dep(d2, t);
        dep(d2, kk);
        dep(d2, jj);
        u.push_back({0, t, kk, jj});
        deps.push_back(d2);
        last[t] = (int)u.size() - 1;
      }
    }
  const int N = (int)u.size();
  std::vector<std::vector<int>> succ(N);
  std::vector<int> pending(N, 0), prio(N, 1);
  for (int i = 0; i < N; i++) {
    std::sort(deps[i].begin(), deps[i].end());
    deps[i].erase(std::unique(deps[i].begin(), deps[i].end()), deps[i].end());
    pending[i] = (int)deps[i].size();
    for (int p : deps[i]) succ[p].push_back(i);
  }
  for (int i = N - 1; i >= 0; i--)
    for (int s : succ[i]) prio[i] = std::max(prio[i], prio[s] + 1);
  std::vector<int> ready;
  for (int i = 0; i < N; i++)
    if (pending[i] == 0) ready.push_back(i);
  CoopStream st;
  int left = N;
  while (left > 0) {
    std::sort(ready.begin(), ready.end(), [&](int a, int b) {
      return prio[a] != prio[b] ? prio[a] > prio[b] : a < b;
    });
    const int kind = u[ready[0]].div;
    std::vector<int> take, keep;
    for (int r : ready)
      if (u[r].div == kind && (int)take.size() < kCoopLuCap * kCoopLanes) take.push_back(r);
      else keep.push_back(r);
    std::vector<int> cnt(kCoopLanes, 0);
    std::vector<int> next;
    // the shortest lane streams take the first units of the iteration
    std::vector<int> order(kCoopLanes);
    for (int l = 0; l < kCoopLanes; l++) order[l] = l;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return st.lane[a].size() < st.lane[b].size(); });
    for (size_t i = 0; i < take.size(); i++) {
      const int l = order[i % kCoopLanes];
      const Unit& x = u[take[i]];
      st.lane[l].push_back((unsigned)x.div << 31 | (unsigned)x.t << (2 * B) |
                           (unsigned)x.mm << B | (unsigned)x.s);
      cnt[l]++;
      left--;
      for (int s : succ[take[i]])
        if (--pending[s] == 0) next.push_back(s);
    }
    st.count.push_back(cnt);
    ready = keep;
    ready.insert(ready.end(), next.begin(), next.end());
  }
  return st;
}

// Forward substitution (L, unit diagonal).  Entry =
// a | c<<B | r<<(B+C) | start<<(B+2C) | end<<(B+2C+1):
// start: acc = X[r]; a term: acc = acc - J[a]*X[c]; end: X[r] = acc.  Each
// row's terms stay on one lane in the row's own order; a row starts once its
// first operand is final, and a term waits for its operand.  (The backward
// substitution is one dependent chain -- every row begins with the row just
// below it -- so the kernel runs it as straight-line code on one lane.)
CoopStream coop_schedule_forward(const Mechanism& m, int B, int C) {
  const int n = m.nvar;
  std::vector<std::vector<std::pair<int, int>>> terms(n);
  for (int r = 0; r < n; r++)
    for (int j = m.lu_crow[r]; j < m.lu_diag[r]; j++) terms[r].push_back({j, m.lu_icol[j]});
  const int INF = 1 << 30;
  std::vector<int> fin(n, INF);
  std::vector<char> started(n, 0);
  int todo = 0;
  for (int r = 0; r < n; r++) {
    if (terms[r].empty()) {
      fin[r] = -1;  // unchanged, final from the start
      started[r] = 1;
    } else {
      todo++;
    }
  }
  // priority: terms still to run on the longest dependency path from the row
  std::vector<std::vector<int>> users(n);
  for (int r = 0; r < n; r++)
    for (auto& t : terms[r]) users[t.second].push_back(r);
  std::vector<int> tail(n, 0);
  for (int r = n - 1; r >= 0; r--) {  // users come after r
    int best = 0;
    for (int w : users[r]) best = std::max(best, tail[w]);
    tail[r] = (int)terms[r].size() + 1 + best;
  }
  std::vector<int> row(kCoopLanes, -1), next_term(kCoopLanes, 0);
  CoopStream st;
  const unsigned S0 = 1u << (B + 2 * C), E0 = 1u << (B + 2 * C + 1);
  for (int it = 0; todo > 0; it++) {
    if (it > 100000) break;  // no progress: cannot happen for a triangular system
    std::vector<int> cnt(kCoopLanes, 0);
    // lanes with the shortest streams pick new rows first
    std::vector<int> order(kCoopLanes);
    for (int l = 0; l < kCoopLanes; l++) order[l] = l;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
      return (row[a] >= 0) != (row[b] >= 0) ? row[a] >= 0 : st.lane[a].size() < st.lane[b].size();
    });
    for (int l : order) {
      while (cnt[l] < kCoopSolveCap) {
        if (row[l] < 0) {
          int best = -1;
          for (int r = 0; r < n; r++) {
            if (started[r]) continue;
            const bool ok = fin[terms[r][0].second] < it;
            if (ok && (best < 0 || tail[r] > tail[best])) best = r;
          }
          if (best < 0) break;
          started[best] = 1;
          row[l] = best;
          next_term[l] = 0;
        }
        const int r = row[l];
        const int k = next_term[l];
        const auto& t = terms[r][k];
        if (fin[t.second] >= it) break;  // operand not final yet
        const bool last = k + 1 == (int)terms[r].size();
        st.lane[l].push_back((unsigned)t.first | (unsigned)t.second << B |
                             (unsigned)r << (B + C) | (k == 0 ? S0 : 0u) | (last ? E0 : 0u));
        cnt[l]++;
        next_term[l]++;
        if (last) {
          fin[r] = it;
          todo--;
          row[l] = -1;
        }
      }
    }
    st.count.push_back(cnt);
  }
  return st;
}

// Sums: each output (a Vdot row or a Jacobian entry) is a left-to-right sum of
// coefficient * product; outputs go to the least loaded lane, longest first.
struct CoopSumLayout {
  int src_bits, coef_bits, dst_bits;
};
std::vector<unsigned> coop_schedule_sums(const std::vector<std::vector<std::pair<int, int>>>& outs,
                                         const std::vector<char>& diag, CoopSumLayout L,
                                         int& per_lane) {
  std::vector<int> idx(outs.size());
  for (size_t i = 0; i < idx.size(); i++) idx[i] = (int)i;
  auto cost = [&](int o) { return std::max<int>(1, (int)outs[o].size()); };
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return cost(a) > cost(b); });
  std::vector<std::vector<int>> lanes(kCoopLanes);
  std::vector<int> load(kCoopLanes, 0);
  for (int o : idx) {
    int l = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    lanes[l].push_back(o);
    load[l] += cost(o);
  }
  CoopStream st;
  const int F = L.src_bits + L.coef_bits;
  for (int l = 0; l < kCoopLanes; l++)
    for (int o : lanes[l]) {
      const unsigned dst = (unsigned)o << (F + 4);
      const unsigned dg = diag[o] ? 1u << (F + 3) : 0u;
      if (outs[o].empty()) {
        st.lane[l].push_back(dst | dg | 1u << (F + 2) | 1u << (F + 1) | 1u << F);
        continue;
      }
      for (size_t k = 0; k < outs[o].size(); k++)
        st.lane[l].push_back(dst | dg | (k + 1 == outs[o].size() ? 1u << (F + 1) : 0u) |
                             (k == 0 ? 1u << F : 0u) |
                             (unsigned)outs[o][k].second << L.src_bits |
                             (unsigned)outs[o][k].first);
    }
  per_lane = (int)st.max_len();
  return st.interleaved(0xFFFFFFFFu);
}

// The tables of csrc/kpp_coop.cuh for mechanism m (KPP_COOP 0 when the
// mechanism exceeds the 32-bit packing: more than 1024 LU entries, 128
// variable species, 255 extended-state entries or four reactant factors).
void emit_coop_tables(std::ostream& o, const Mechanism& m) {
  View vw(m);
  const int nvar = m.nvar, nr = m.nreact();
  const int next = m.nvar + m.nfix + 1;  // V, FIX, 1.0
  const int ONE = m.nvar + m.nfix;
  auto factors = [&](int eq, int skip, std::vector<int>& out) {
    for (int i = 0; i < nvar; i++) {
      int k = (int)vw.left(i, eq) - (i == skip ? 1 : 0);
      for (int c = 0; c < k; c++) out.push_back(i);
    }
    for (int i = nvar; i < m.nspec; i++)
      for (int c = 0; c < (int)vw.left(i, eq); c++) out.push_back(i);
  };
  // constants: 1.0 first, then the sums' coefficients, then weight constants
  std::vector<double> kc{1.0};
  auto code = [&](double v) {
    for (size_t i = 0; i < kc.size(); i++)
      if (std::memcmp(&kc[i], &v, sizeof v) == 0) return (int)i;
    kc.push_back(v);
    return (int)kc.size() - 1;
  };
  // products of Fun (A, one per equation that changes a variable species) and
  // of Jac_SP (B, one per reactant occurrence), with their weights
  struct Prod { int rct; double k1, k2; std::vector<int> f; };
  std::vector<Prod> pa, pb;
  std::vector<int> a_of_eq(nr, -1);
  int maxf = 1;
  for (int j = 0; j < nr; j++) {
    bool used = false;
    for (int i = 0; i < nvar; i++)
      if (vw.net(i, j) != 0) { used = true; break; }
    if (!used) continue;
    Head h = head_of(m, j, 1.0f);
    Prod p{h.rct, h.k1, h.k2, {}};
    factors(j, -1, p.f);
    maxf = std::max(maxf, (int)p.f.size());
    a_of_eq[j] = (int)pa.size();
    pa.push_back(p);
  }
  std::vector<std::vector<int>> bidx(nr, std::vector<int>(nvar, -1));
  for (int i = 0; i < nr; i++)
    for (int j = 0; j < nvar; j++) {
      if (vw.left(j, i) == 0) continue;
      bidx[i][j] = (int)pb.size();
      Head h = head_of(m, i, vw.left(j, i));
      Prod p{h.rct, h.k1, h.k2, {}};
      factors(i, j, p.f);
      maxf = std::max(maxf, (int)p.f.size());
      pb.push_back(p);
    }
  // sums: Vdot rows over A, Jacobian entries (LU pattern) over B
  std::vector<std::vector<std::pair<int, int>>> vsum(nvar), jsum;
  std::vector<char> vdiag(nvar, 0), jdiag;
  for (int i = 0; i < nvar; i++)
    for (int j = 0; j < nr; j++) {
      const float c = vw.net(i, j);
      if (c != 0) vsum[i].push_back({a_of_eq[j], code(const_value(c))});
    }
  for (int i = 0; i < nvar; i++)
    for (int j = 0; j < nvar; j++) {
      if (!(m.lustruct[i][j] || i == j)) continue;
      std::vector<std::pair<int, int>> t;
      if (m.lustruct[i][j])
        for (int k = 0; k < nr; k++)
          if (vw.net(i, k) * (bidx[k][j] >= 0 ? 1.0f : 0.0f) != 0)
            t.push_back({bidx[k][j], code(const_value(vw.net(i, k)))});
      jsum.push_back(t);
      jdiag.push_back(i == j);
    }
  const int nsumcoef = (int)kc.size();  // codes of the sums' coefficients come first
  std::vector<unsigned> wa, wb;  // weight words: rct | k1 code | k2 code
  const int RB = bits_for(nr + 1);
  auto weights = [&](const std::vector<Prod>& ps, std::vector<unsigned>& out) {
    for (const Prod& p : ps)
      out.push_back((unsigned)(p.rct >= 0 ? p.rct : nr) | (unsigned)code(p.k1) << RB |
                    (unsigned)code(p.k2) << (RB + 12));
  };
  weights(pa, wa);
  weights(pb, wb);
  const int ncoef = (int)kc.size();  // every constant, the weights' included
  const int B = bits_for(m.lu_nonzero), C = bits_for(nvar);
  CoopSumLayout SL{bits_for(std::max<size_t>({pa.size(), pb.size(), 2})), bits_for(nsumcoef),
                   bits_for(std::max(m.lu_nonzero, nvar))};
  const bool fits = m.lu_nonzero <= 1024 && nvar <= 128 && next <= 255 && maxf <= 4 &&
                    (long)kc.size() <= 4096 && RB + 24 <= 32 &&
                    SL.src_bits + SL.coef_bits + 4 + SL.dst_bits <= 32 &&
                    B + 2 * C + 3 <= 32;
  o << "\n// ---- tables of the warp-per-cell kernel (csrc/kpp_coop.cuh) ----\n";
  if (!fits) {
    o << "#define KPP_COOP 0\n";
    return;
  }
  o << "#define KPP_COOP 1\nnamespace kpp_coop {\n";
  auto prod_words = [&](const std::vector<Prod>& ps) {
    const size_t rounds = (ps.size() + kCoopLanes - 1) / kCoopLanes;
    std::vector<unsigned> out(rounds * kCoopLanes, 0);
    for (size_t t = 0; t < out.size(); t++) {
      unsigned w = 0;
      for (int f = 0; f < 4; f++) {
        const int idx = (t < ps.size() && f < (int)ps[t].f.size()) ? ps[t].f[f] : ONE;
        w |= (unsigned)idx << (8 * f);
      }
      out[t] = w;
    }
    return out;
  };
  std::vector<unsigned> fa = prod_words(pa), fb = prod_words(pb);
  wa.resize(fa.size(), (unsigned)nr);
  wb.resize(fb.size(), (unsigned)nr);
  int lv = 0, lj = 0;
  std::vector<unsigned> sv = coop_schedule_sums(vsum, vdiag, SL, lv);
  std::vector<unsigned> sj = coop_schedule_sums(jsum, jdiag, SL, lj);
  CoopStream lu = coop_schedule_lu(m, B);
  CoopStream fw = coop_schedule_forward(m, B, C);
  std::vector<unsigned> diag(m.lu_diag.begin(), m.lu_diag.begin() + nvar);
  struct Part { const char* name; std::vector<unsigned> words; };
  std::vector<Part> parts = {
      {"PF", fa}, {"WF", wa}, {"PJ", fb}, {"WJ", wb}, {"SV", sv}, {"SJ", sj},
      {"CLU", lu.counts()}, {"LU", lu.interleaved(0)}, {"CFW", fw.counts()},
      {"FW", fw.interleaved(0)}, {"DIAG", diag}};
  long total_words = 0;
  for (auto& p : parts) total_words += (long)p.words.size();
  // one cell of the six-stage method beside the tables must fit the 227 KB of
  // shared memory a CTA can hold, and the rate constants are staged in the
  // cell's matrix and product area
  const long cell6 = 2L * next + 9L * nvar + m.lu_nonzero + (long)pa.size() +
                     ((long)pb.size() > 7L * nvar ? (long)pb.size() : 0L);
  const long table_bytes = (total_words * 4 + 15) / 16 * 16 + 8L * ncoef;
  if (table_bytes + 8 * cell6 > 227L * 1024 || m.lu_nonzero + (long)pa.size() < nr) {
    o << "}  // namespace kpp_coop\n#undef KPP_COOP\n#define KPP_COOP 0\n";
    return;
  }
  long off = 0;
  std::vector<unsigned> all;
  for (auto& p : parts) {
    o << "constexpr int O_" << p.name << " = " << off << ";\n";
    off += (long)p.words.size();
    all.insert(all.end(), p.words.begin(), p.words.end());
  }
  long sum_terms_v = 0, sum_terms_j = 0;
  for (auto& s : vsum) sum_terms_v += (long)s.size();
  for (auto& s : jsum) sum_terms_j += (long)s.size();
  o << "constexpr int TAB_WORDS = " << off << ";\n"
    << "constexpr int NEXT = " << next << ", ONE = " << ONE << ";\n"
    << "constexpr int NA = " << pa.size() << ", NB = " << pb.size() << ", MAXF = " << maxf
    << ";\n"
    << "constexpr int RF = " << fa.size() / kCoopLanes << ", RJ = " << fb.size() / kCoopLanes
    << ";  // product rounds\n"
    << "constexpr int NKC = " << ncoef << ";\n"
    << "constexpr int RATE_BITS = " << RB << ", NO_RATE = " << nr << ";\n"
    << "constexpr int SUM_SRC_BITS = " << SL.src_bits << ", SUM_COEF_BITS = " << SL.coef_bits
    << ";\n"
    << "constexpr int LV = " << lv << ", LJ = " << lj << ";  // entries per lane of the sums ("
    << sum_terms_v << " and " << sum_terms_j << " terms)\n"
    << "constexpr int IT_LU = " << lu.count.size() << ", IT_FW = " << fw.count.size()
    << ";  // iterations\n"
    << "constexpr int LU_BITS = " << B << ", X_BITS = " << C << ";\n"
    << "constexpr int LU_CAP = " << kCoopLuCap << ", SOLVE_CAP = " << kCoopSolveCap
    << ";  // entries per lane per iteration\n";
  emit_table(o, "unsigned int", "tab", all);
  emit_dtable(o, "kc", kc);
  o << "}  // namespace kpp_coop\n";
}

}  // namespace

// Host-side files of a mechanism:
//   <prefix>_host.h        the user-to-KPP species map of the C ABI's
//                          shuffle entries (GenerateShuffle_user2kpp /
//                          _kpp2user, src/gen.c:3401-3468): user species k is
//                          the k-th species declared variable (after #SETFIX)
//                          among declaration codes 1 .. NSPEC-1, unused ones
//                          counted, and only k < NVAR are mapped (initNr =
//                          VarNr, src/kpp.c:594)
//   <prefix>_Parameters.h  sizes and species indices for a host model in C
//                          (the generated ROOT_Parameters.h, src/gen.c:2627-2720)
bool emit_host(const Mechanism& m, const std::string& out_prefix) {
  View vw(m);
  const int nvar = m.nvar, nspec = m.nspec;
  std::vector<int> final_of_slot(m.order.size(), -1);
  for (int f = 0; f < nspec; f++) final_of_slot[m.spc_slot[f]] = f;
  // The reference visits declaration codes 1 .. SpcNr-1 only, SpcNr being
  // the number of species that take part (NSPEC): with unused declared
  // species the last declarations are never reached.
  std::vector<int> user;
  for (int i = 1; i < std::min((int)m.table.size(), nspec); i++) {
    if (m.table[i].type != SPC_VAR) continue;
    auto it = m.slot_of_code.find(i);
    int f = it == m.slot_of_code.end() ? -1 : final_of_slot[it->second];
    user.push_back(((int)user.size() < nvar && f >= 0) ? f : -1);
  }
  {
    std::ostringstream o;
    o << "// Generated by kppcu.  Do not edit.  Host data of mechanism " << m.root << ".\n"
      << "#pragma once\n\n#define KPP_NUSER " << user.size() << "\n\n"
      << "namespace kpp_host {\n";
    emit_int_table(o, "kUserToKpp", user);
    o << "}  // namespace kpp_host\n";
    std::ofstream f(out_prefix + "_host.h");
    if (!f) return false;
    f << o.str();
  }
  {
    std::ostringstream o;
    o << "/* Generated by kppcu.  Do not edit.  Sizes and species indices of mechanism\n"
      << "   " << m.root << " (KPP's ROOT_Parameters.h) for host models. */\n"
      << "#ifndef KPP_B200_" << m.root << "_PARAMETERS_H\n"
      << "#define KPP_B200_" << m.root << "_PARAMETERS_H\n\n"
      << "#define NSPEC " << nspec << "\n#define NVAR " << nvar << "\n#define NVARACT "
      << m.nvaract << "\n#define NFIX " << (m.nfix > 0 ? m.nfix : 1) << "\n#define NREACT "
      << m.nreact() << "\n#define NVARST 0\n#define NFIXST " << nvar << "\n#define NONZERO "
      << m.nonzero << "\n#define LU_NONZERO " << m.lu_nonzero << "\n#define CNVAR " << nvar + 1
      << "\n\n";
    for (int i = 0; i < nspec; i++) o << "#define ind_" << vw.name(i) << " " << i << "\n";
    for (int i = nvar; i < nspec; i++) o << "#define indf_" << vw.name(i) << " " << (i - nvar) << "\n";
    o << "\n#endif\n";
    std::ofstream f(out_prefix + "_Parameters.h");
    if (!f) return false;
    f << o.str();
  }
  return true;
}

bool emit_cuda(const Mechanism& m, const std::string& out_prefix) {
  View vw(m);
  long ops_fun = 0, ops_jac = 0, ops_decomp = 0, ops_solve = 0;
  const int nvar = m.nvar, nfix = m.nfix, nspec = m.nspec, nr = m.nreact();
  std::ostringstream o;

  o << "// Generated by kppcu, the KPP mechanism compiler of kpp_b200.  Do not edit.\n"
    << "// Mechanism: " << m.root << "\n"
    << "#pragma once\n\n"
    << "#define KPP_MECH_NAME " << c_string(m.root) << "\n"
    << "#define KPP_NVAR " << nvar << "\n"
    << "#define KPP_NFIX " << (nfix > 0 ? nfix : 1) << "\n"
    << "#define KPP_NFIX_TRUE " << nfix << "\n"
    << "#define KPP_NSPEC " << nspec << "\n"
    << "#define KPP_NVARACT " << m.nvaract << "\n"
    << "#define KPP_NREACT " << nr << "\n"
    << "#define KPP_NONZERO " << m.nonzero << "\n"
    << "#define KPP_LU_NONZERO " << m.lu_nonzero << "\n"
    << "#define KPP_CFACTOR " << std::to_string(m.cfactor) << "\n\n";
  {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.17g", m.cfactor);
    o << "#undef KPP_CFACTOR\n#define KPP_CFACTOR " << buf << "\n\n";
  }
  o << "// Large mechanisms call their unrolled rate, Fun, Jac_SP, LU and solve\n"
       "// functions instead of inlining every call site: compile time grows with\n"
       "// each inlined copy of a body of tens of thousands of operations, and one\n"
       "// call is negligible next to such a body.\n"
       "#ifndef KPP_MECH_INLINE\n"
    << "#define KPP_MECH_INLINE " << (m.lu_nonzero >= kGenericLu ? "__noinline__" : "__forceinline__")
    << "\n#endif\n\n";
  o << "// Species indices (variable species first, then fixed species).\n";
  for (int i = 0; i < nspec; i++) o << "#define ind_" << vw.name(i) << " " << i << "\n";
  for (int i = nvar; i < nspec; i++) o << "#define indf_" << vw.name(i) << " " << (i - nvar) << "\n";
  o << "\n";

  // ---- host/device tables
  o << "namespace kpp_mech {\n\n";
  o << "static const char* const kSpeciesNames[" << nspec << "] = {";
  for (int i = 0; i < nspec; i++) o << (i % 6 == 0 ? "\n    " : " ") << c_string(vw.name(i)) << ",";
  o << "};\n\n";
  o << "// #INITVALUES, before the CFACTOR scaling (values in mechanism units)\n";
  o << "static const double kInitialValues[" << nspec << "] = {";
  for (int i = 0; i < nspec; i++) {
    const Species& s = m.table[m.order[m.spc_slot[i]]];
    std::string v = !s.ival.empty() ? s.ival : (i < nvar ? m.var_default : m.fix_default);
    for (char& ch : v)
      if (ch == 'd' || ch == 'D') ch = 'e';
    o << (i % 6 == 0 ? "\n    " : " ") << "(" << v << "),";
  }
  o << "};\n\n";
  emit_int_table(o, "kLuIRow", m.lu_irow);
  emit_int_table(o, "kLuICol", m.lu_icol);
  emit_int_table(o, "kLuCRow", m.lu_crow);
  emit_int_table(o, "kLuDiag", m.lu_diag);
  o << "\n";
  std::vector<int> kinds;
  for (const Reaction& r : m.reactions) kinds.push_back((int)r.kind);
  emit_int_table(o, "kRateKind", kinds);
  o << "\n}  // namespace kpp_mech\n\n";

  // ---- user device code from the CUDA_* inline blocks
  for (const char* ctx : {"CUDA_GLOBAL", "CUDA_UTIL", "CUDA_RATES"}) {
    auto it = m.inline_code.find(ctx);
    if (it != m.inline_code.end()) o << "// #INLINE " << ctx << "\n" << it->second << "\n";
  }

  // ---- rate constants, split by what they depend on
  // Every rate is recomputed from the same inputs wherever the reference
  // recomputes it, so hoisting a rate out of the time loop when its inputs
  // are constant for the cell gives the same bits.
  std::vector<int> rclass(nr, RC_STATIC);
  // Inline rate prologues: CUDA_RCONST_STATIC (depends on TEMP / CFACTOR
  // only) and CUDA_RCONST_SUN (also on SUN) declare names a rate may use
  // without leaving that class; CUDA_RCONST alone (code of unknown
  // dependence) makes every rate dynamic.
  auto inl = [&](const char* k) {
    auto it = m.inline_code.find(k);
    return it == m.inline_code.end() ? std::string() : it->second;
  };
  const std::string inl_static = inl("CUDA_RCONST_STATIC"), inl_sun = inl("CUDA_RCONST_SUN"),
                    inl_dyn = inl("CUDA_RCONST");
  const bool classed = !inl_static.empty() || !inl_sun.empty();
  const bool rconst_inline = !inl_dyn.empty() && !classed;
  const std::set<std::string> static_names = declared_names(inl_static);
  const std::set<std::string> sun_names = declared_names(inl_sun);
  for (int j = 0; j < nr; j++) {
    const Reaction& r = m.reactions[j];
    if (r.kind == RATE_NUMBER) { rclass[j] = -1; continue; }
    rclass[j] = rconst_inline ? RC_DYNAMIC : classify_rate(r.rate, static_names, sun_names);
  }
  const char* kRateMacros =
      "#define ARR_abc(a0, b0, c0) kpp_arr_abc(TEMP, (float)(a0), (float)(b0), (float)(c0))\n"
      "#define ARR_ab(a0, b0) kpp_arr_ab(TEMP, (float)(a0), (float)(b0))\n"
      "#define ARR_ac(a0, c0) kpp_arr_ac(TEMP, (float)(a0), (float)(c0))\n"
      "#define EP2(a0, c0, a2, c2, a3, c3) kpp_ep2(TEMP, CFACTOR, (float)(a0), (float)(c0), "
      "(float)(a2), (float)(c2), (float)(a3), (float)(c3))\n"
      "#define EP3(a1, c1, a2, c2) kpp_ep3(TEMP, CFACTOR, (float)(a1), (float)(c1), (float)(a2), "
      "(float)(c2))\n"
      "#define FALL(a0, b0, c0, a1, b1, c1, cf) kpp_fall(TEMP, CFACTOR, (float)(a0), (float)(b0), "
      "(float)(c0), (float)(a1), (float)(b1), (float)(c1), (float)(cf))\n";
  const char* kRateUndef = "#undef ARR_abc\n#undef ARR_ab\n#undef ARR_ac\n#undef EP2\n#undef EP3\n#undef FALL\n";
  int ncls[3] = {0, 0, 0};
  for (int j = 0; j < nr; j++)
    if (rclass[j] >= 0) ncls[rclass[j]]++;
  o << "// Rate constants by dependence: " << ncls[RC_STATIC] << " depend only on TEMP and CFACTOR,\n"
    << "// " << ncls[RC_SUN] << " also on SUN, " << ncls[RC_DYNAMIC]
    << " on the time or the concentrations.\n"
    << "#define KPP_RATES_SUN " << ncls[RC_SUN] << "\n"
    << "#define KPP_RATES_DYNAMIC " << ncls[RC_DYNAMIC] << "\n\n";
  // The arithmetic (rates, Fun, Jac_SP, LU, solve) can come from KPP's own
  // generator instead (kpp_b200/kppgen: #LANGUAGE CUDA); such a build defines
  // KPP_EXTERNAL_ARITHMETIC and supplies these functions itself.
  o << "#ifndef KPP_EXTERNAL_ARITHMETIC\n";
  const char* names[3] = {"kpp_rconst_static", "kpp_rconst_sun", "kpp_rconst_dynamic"};
  for (int c = 0; c < 3; c++) {
    o << "template <class TR, class TV, class TF>\n"
      << "__device__ KPP_MECH_INLINE void " << names[c]
      << "(TR& RCONST, const double TIME, const double TEMP, const double CFACTOR,\n"
         "    double SUN, const TV& VAR, const TF& FIX) {\n"
         "  (void)TIME; (void)TEMP; (void)CFACTOR; (void)SUN; (void)VAR; (void)FIX;\n"
      << kRateMacros;
    if (!inl_static.empty()) o << "  // #INLINE CUDA_RCONST_STATIC\n" << inl_static << "\n";
    if (c >= RC_SUN && !inl_sun.empty()) o << "  // #INLINE CUDA_RCONST_SUN\n" << inl_sun << "\n";
    if (c == RC_DYNAMIC && !inl_dyn.empty()) o << "  // #INLINE CUDA_RCONST\n" << inl_dyn << "\n";
    for (int j = 0; j < nr; j++) {
      if (rclass[j] == c) o << "  RCONST[" << j << "] = (" << m.reactions[j].rate << ");\n";
      // constant rates are folded into Fun/Jac_SP; the reference's
      // Initialize() also stores them in RCONST (as single-precision values)
      if (c == RC_STATIC && rclass[j] < 0)
        o << "  RCONST[" << j << "] = " << fmt_g(m.reactions[j].number) << ";\n";
    }
    o << kRateUndef << "}\n\n";
  }
  o << "// All rate constants at time TIME (Update_RCONST, src/gen.c:2343-2473).\n"
       "template <class TR, class TV, class TF>\n"
       "__device__ __forceinline__ void kpp_update_rconst(TR& RCONST, const double TIME,\n"
       "    const double TEMP, const double CFACTOR, double SUN, const TV& VAR, const TF& FIX) {\n"
       "  kpp_rconst_static(RCONST, TIME, TEMP, CFACTOR, SUN, VAR, FIX);\n"
       "  kpp_rconst_sun(RCONST, TIME, TEMP, CFACTOR, SUN, VAR, FIX);\n"
       "  kpp_rconst_dynamic(RCONST, TIME, TEMP, CFACTOR, SUN, VAR, FIX);\n"
       "}\n\n";

  // ---- Fun (aggregate form)
  o << "// ODE right-hand side Vdot = f(V) of one cell; A holds the equation rates.\n"
       "template <class TV, class TF, class TR, class TO, class TA>\n"
       "__device__ KPP_MECH_INLINE void kpp_fun(const TV& V, const TF& F, const TR& RCT,\n"
       "    TO& Vdot, TA& A) {\n"
       "  (void)F; (void)RCT;\n";
  for (int j = 0; j < nr; j++) {
    bool used = false;
    for (int i = 0; i < nvar; i++)
      if (vw.net(i, j) != 0) { used = true; break; }
    if (!used) continue;
    P prod = vw.reactants(vw.rconst(j), j, -1);
    ops_fun += count_ops(prod);
    o << "  A[" << j << "] = " << print(prod) << ";\n";
  }
  for (int i = 0; i < nvar; i++) {
    P sum = cnst(0);
    for (int j = 0; j < nr; j++) sum = add(sum, mul(cnst(vw.net(i, j)), leaf("A[" + std::to_string(j) + "]")));
    ops_fun += count_ops(sum);
    o << "  Vdot[" << i << "] = " << print(sum) << ";\n";
  }
  o << "}\n#endif  // KPP_EXTERNAL_ARITHMETIC\n\n";

  // ---- Jac_SP
  std::vector<std::vector<int>> bidx(nr, std::vector<int>(nvar, -1));
  int nb = 0;
  for (int i = 0; i < nr; i++)
    for (int j = 0; j < nvar; j++)
      if (vw.left(j, i) != 0) bidx[i][j] = nb++;
  o << "#define KPP_NJAC_TMP " << (nb > 0 ? nb : 1) << "\n\n#ifndef KPP_EXTERNAL_ARITHMETIC\n";
  o << "// Sparse Jacobian of one cell in the LU pattern (fill-in entries are 0);\n"
       "// NEG = true writes its negation (the -Jac0 of ros_PrepareMatrix).  B holds\n"
       "// the partial derivatives of the equation rates (KPP_NJAC_TMP entries).\n"
       "template <bool NEG, class TV, class TF, class TR, class TJ, class TB>\n"
       "__device__ KPP_MECH_INLINE void kpp_jac_sp(const TV& V, const TF& F, const TR& RCT,\n"
       "    TJ& JVS, TB& B) {\n"
       "  (void)V; (void)F; (void)RCT;\n";
  for (int i = 0; i < nr; i++)
    for (int j = 0; j < nvar; j++) {
      if (bidx[i][j] < 0) continue;
      P prod = mul(vw.rconst(i), cnst(vw.left(j, i)));
      prod = vw.reactants(prod, i, j);
      ops_jac += count_ops(prod);
      o << "  B[" << bidx[i][j] << "] = " << print(prod) << ";\n";
    }
  {
    int n = 0;
    for (int i = 0; i < nvar; i++)
      for (int j = 0; j < nvar; j++) {
        if (m.lustruct[i][j]) {
          P sum = cnst(0);
          for (int k = 0; k < nr; k++)
            if (vw.net(i, k) * (bidx[k][j] >= 0 ? 1.0f : 0.0f) != 0)
              sum = add(sum, mul(cnst(vw.net(i, k)), leaf("B[" + std::to_string(bidx[k][j]) + "]")));
          ops_jac += count_ops(sum);
          o << "  JVS[" << n << "] = NEG ? -(" << print(sum) << ") : (" << print(sum) << ");\n";
          n++;
        } else if (i == j) {
          o << "  JVS[" << n << "] = NEG ? -0.0 : 0.0;\n";
          n++;
        }
      }
  }
  o << "}\n\n";

  // ---- diagonal shift of ros_PrepareMatrix (int/rosenbrock.c:720-723)
  o << "// JVS[diag] += v for every row (the 1/(h*gamma) shift of the Rosenbrock matrix).\n"
       "template <class TJ>\n"
       "__device__ __forceinline__ void kpp_add_diagonal(TJ& JVS, const double v) {\n";
  for (int i = 0; i < nvar; i++)
    o << "  JVS[" << m.lu_diag[i] << "] = JVS[" << m.lu_diag[i] << "] + v;\n";
  o << "}\n#endif  // KPP_EXTERNAL_ARITHMETIC\n\n";

  // ---- KppDecomp and KppSolve.  Mechanisms below kGenericLu LU entries get
  // both fully unrolled; larger ones (MCM isoprene: 7123 entries, a 41k
  // operation LU) get the reference's own loops over the LU tables (in
  // constant memory, read uniformly by a warp), the same operations in the
  // same order: an unrolled body of tens of thousands of operations takes the
  // device compiler many minutes per translation unit and runs from the
  // instruction cache poorly.
  const bool generic_lu = m.lu_nonzero >= kGenericLu;
  if (generic_lu) {
    auto table = [&](const char* name, const std::vector<int>& v) {
      o << "__constant__ int " << name << "[" << v.size() << "] = {";
      for (size_t i = 0; i < v.size(); i++) o << (i % 16 == 0 ? "\n    " : " ") << v[i] << ",";
      o << "};\n";
    };
    o << "#define KPP_LU_GENERIC 1\n";
    table("kpp_lu_crow_c", m.lu_crow);
    table("kpp_lu_diag_c", m.lu_diag);
    table("kpp_lu_icol_c", m.lu_icol);
    for (int k = 0; k < nvar; k++)
      for (int kk = m.lu_crow[k]; kk < m.lu_diag[k]; kk++) {
        const int j = m.lu_icol[kk];
        ops_decomp += 1 + 2L * (m.lu_crow[j + 1] - m.lu_diag[j] - 1);
      }
    for (int i = 0; i < nvar; i++)
      ops_solve += 2L * (m.lu_crow[i + 1] - m.lu_crow[i] - 1) + 1;
    o << "\n#ifndef KPP_EXTERNAL_ARITHMETIC\n"
         "// In-place no-pivot sparse LU of one cell (KppDecomp, util/sutil.c:2-23), row by\n"
         "// row through the dense work row W of NVAR entries; returns k+1 when the\n"
         "// diagonal entry of row k is zero on entry to its elimination, 0 on success.\n"
         "template <class TJ, class TW>\n"
         "__device__ __noinline__ int kpp_decomp(TJ& JVS, TW& W) {\n"
         "  for (int k = 0; k < KPP_NVAR; k++) {\n"
         "    const int dk = kpp_lu_diag_c[k], b = kpp_lu_crow_c[k], e = kpp_lu_crow_c[k + 1];\n"
         "    if (JVS[dk] == 0.0) return k + 1;\n"
         "    for (int kk = b; kk < e; kk++) W[kpp_lu_icol_c[kk]] = JVS[kk];\n"
         "    for (int kk = b; kk < dk; kk++) {\n"
         "      const int j = kpp_lu_icol_c[kk];\n"
         "      const double a = -W[j] / JVS[kpp_lu_diag_c[j]];\n"
         "      W[j] = -a;\n"
         "      for (int jj = kpp_lu_diag_c[j] + 1; jj < kpp_lu_crow_c[j + 1]; jj++) {\n"
         "        const int c = kpp_lu_icol_c[jj];\n"
         "        W[c] = W[c] + a*JVS[jj];\n"
         "      }\n"
         "    }\n"
         "    for (int kk = b; kk < e; kk++) JVS[kk] = W[kpp_lu_icol_c[kk]];\n"
         "  }\n"
         "  return 0;\n"
         "}\n\n"
         "// Solve (LU) x = b in place, b given in X (KppSolve, src/gen.c:1960-2034: each\n"
         "// row's terms subtracted left to right, the backward rows divided last).\n"
         "template <class TJ, class TX>\n"
         "__device__ __noinline__ void kpp_solve(const TJ& JVS, TX& X) {\n"
         "  for (int i = 0; i < KPP_NVAR; i++) {\n"
         "    const int b = kpp_lu_crow_c[i], d = kpp_lu_diag_c[i];\n"
         "    if (b < d) {\n"
         "      double x = X[i];\n"
         "      for (int j = b; j < d; j++) x = x - JVS[j]*X[kpp_lu_icol_c[j]];\n"
         "      X[i] = x;\n"
         "    }\n"
         "  }\n"
         "  for (int i = KPP_NVAR - 1; i >= 0; i--) {\n"
         "    const int d = kpp_lu_diag_c[i];\n"
         "    double x = X[i];\n"
         "    for (int j = d + 1; j < kpp_lu_crow_c[i + 1]; j++) x = x - JVS[j]*X[kpp_lu_icol_c[j]];\n"
         "    X[i] = x/JVS[d];\n"
         "  }\n"
         "}\n#endif  // KPP_EXTERNAL_ARITHMETIC\n\n";
  } else {
    std::vector<std::vector<int>> pos(nvar, std::vector<int>(nvar, -1));
    for (int k = 0; k < m.lu_nonzero; k++) pos[m.lu_irow[k]][m.lu_icol[k]] = k;
    o << "#ifndef KPP_EXTERNAL_ARITHMETIC\n"
         "// In-place no-pivot sparse LU of one cell (KppDecomp, util/sutil.c:2-23,\n"
         "// unrolled in its operation order); returns k+1 when the diagonal entry of\n"
         "// row k is zero on entry to its elimination, 0 on success.  W (a work row\n"
         "// for the loop form of large mechanisms) is not used.\n"
         "template <class TJ, class TW>\n"
         "__device__ KPP_MECH_INLINE int kpp_decomp(TJ& JVS, TW& W) {\n"
         "  (void)W;\n"
         "  double a;\n";
    for (int k = 0; k < nvar; k++) {
      o << "  if (JVS[" << m.lu_diag[k] << "] == 0.0) return " << (k + 1) << ";\n";
      for (int kk = m.lu_crow[k]; kk < m.lu_diag[k]; kk++) {
        int j = m.lu_icol[kk];
        ops_decomp += 1;
        o << "  a = -JVS[" << kk << "] / JVS[" << m.lu_diag[j] << "];\n";
        o << "  JVS[" << kk << "] = -a;\n";
        for (int jj = m.lu_diag[j] + 1; jj < m.lu_crow[j + 1]; jj++) {
          int t = pos[k][m.lu_icol[jj]];
          ops_decomp += 2;
          o << "  JVS[" << t << "] = JVS[" << t << "] + a*JVS[" << jj << "];\n";
        }
      }
    }
    o << "  (void)a;\n  return 0;\n}\n\n";

    // ---- KppSolve, unrolled: the forward and the backward substitution as
    // functions of their own (the warp-per-cell kernel runs the backward one
    // on a single lane), and kpp_solve = both
    o << "// Forward substitution of KppSolve in place (L x = b, unit diagonal).\n"
         "template <class TJ, class TX>\n"
         "__device__ KPP_MECH_INLINE void kpp_solve_fw(const TJ& JVS, TX& X) {\n";
    for (int i = 0; i < nvar; i++) {
      int b = m.lu_crow[i], e = m.lu_diag[i];
      if (b < e) {
        P sum = leaf("X[" + std::to_string(i) + "]");
        for (int j = b; j < e; j++)
          sum = sub(sum, mul(leaf("JVS[" + std::to_string(j) + "]"),
                             leaf("X[" + std::to_string(m.lu_icol[j]) + "]")));
        ops_solve += count_ops(sum);
        o << "  X[" << i << "] = " << print(sum) << ";\n";
      }
    }
    o << "}\n\n"
         "// Backward substitution of KppSolve in place (U x = b).\n"
         "template <class TJ, class TX>\n"
         "__device__ KPP_MECH_INLINE void kpp_solve_bw(const TJ& JVS, TX& X) {\n";
    for (int i = nvar - 1; i >= 0; i--) {
      P sum = leaf("X[" + std::to_string(i) + "]");
      for (int j = m.lu_diag[i] + 1; j < m.lu_crow[i + 1]; j++)
        sum = sub(sum, mul(leaf("JVS[" + std::to_string(j) + "]"),
                           leaf("X[" + std::to_string(m.lu_icol[j]) + "]")));
      sum = divide(sum, leaf("JVS[" + std::to_string(m.lu_diag[i]) + "]"));
      ops_solve += count_ops(sum);
      o << "  X[" << i << "] = " << print(sum) << ";\n";
    }
    o << "}\n\n"
         "// Solve (LU) x = b in place, b given in X.\n"
         "template <class TJ, class TX>\n"
         "__device__ __forceinline__ void kpp_solve(const TJ& JVS, TX& X) {\n"
         "  kpp_solve_fw(JVS, X);\n"
         "  kpp_solve_bw(JVS, X);\n"
         "}\n#endif  // KPP_EXTERNAL_ARITHMETIC\n\n";
  }

  // ---- KppDecompCmplxR / KppSolveCmplxR (util/sutil.c:28-90), unrolled.
  // The reference runs these generic loops over LU_CROW / LU_ICOL / LU_DIAG
  // with a dense work row; the elimination reads only row k's own pattern
  // entries and the finished rows above it, so working in place on row k
  // performs the same operations on the same values.
  long ops_decomp_c = 0, ops_solve_c = 0;
  std::ostringstream oc;  // written to <prefix>_cmplx.cuh
  if (m.lu_nonzero >= kGenericLu) {
    // Large patterns: the generic loops over the LU tables, with the dense
    // work row of the reference (the unrolled form would take another long
    // device compile); the same operations in the same order.
    // the LU tables of the mechanism header (kpp_lu_*_c, the real LU's loop form)
    oc << "#define KPP_CMPLX_GENERIC 1\n";
    for (int k = 0; k < nvar; k++)
      for (int kk = m.lu_crow[k]; kk < m.lu_diag[k]; kk++) {
        const int j = m.lu_icol[kk];
        ops_decomp_c += 11 + 8L * (m.lu_crow[j + 1] - m.lu_diag[j] - 1);
      }
    for (int i = 0; i < nvar; i++) ops_solve_c += 8L * (m.lu_crow[i + 1] - m.lu_crow[i] - 1) + 11;
    oc << "\n"
       "// In-place no-pivot sparse LU of the complex matrix (JR + i JI) of one cell,\n"
       "// row by row through the dense work row (WR, WI) of NVAR entries; returns\n"
       "// k+1 when the real or the imaginary part of row k's diagonal entry is zero\n"
       "// on entry to its elimination, 0 on success.\n"
       "template <class TJ, class TW>\n"
       "__device__ __noinline__ int kpp_decomp_cmplx_w(TJ& JR, TJ& JI, TW& WR, TW& WI) {\n"
       "  for (int k = 0; k < KPP_NVAR; k++) {\n"
       "    const int dk = kpp_lu_diag_c[k], b = kpp_lu_crow_c[k], e = kpp_lu_crow_c[k + 1];\n"
       "    if (JR[dk] == 0.0) return k + 1;\n"
       "    if (JI[dk] == 0.0) return k + 1;\n"
       "    for (int kk = b; kk < e; kk++) {\n"
       "      WR[kpp_lu_icol_c[kk]] = JR[kk];\n"
       "      WI[kpp_lu_icol_c[kk]] = JI[kk];\n"
       "    }\n"
       "    for (int kk = b; kk < dk; kk++) {\n"
       "      const int j = kpp_lu_icol_c[kk], dj = kpp_lu_diag_c[j];\n"
       "      const double den = JR[dj]*JR[dj] + JI[dj]*JI[dj];\n"
       "      const double ar = -(WR[j]*JR[dj] + WI[j]*JI[dj])/den;\n"
       "      const double ai = -(WI[j]*JR[dj] - WR[j]*JI[dj])/den;\n"
       "      WR[j] = -ar;\n"
       "      WI[j] = -ai;\n"
       "      for (int jj = dj + 1; jj < kpp_lu_crow_c[j + 1]; jj++) {\n"
       "        const int c = kpp_lu_icol_c[jj];\n"
       "        WR[c] = WR[c] + ar*JR[jj] - ai*JI[jj];\n"
       "        WI[c] = WI[c] + ar*JI[jj] + ai*JR[jj];\n"
       "      }\n"
       "    }\n"
       "    for (int kk = b; kk < e; kk++) {\n"
       "      JR[kk] = WR[kpp_lu_icol_c[kk]];\n"
       "      JI[kk] = WI[kpp_lu_icol_c[kk]];\n"
       "    }\n"
       "  }\n"
       "  return 0;\n"
       "}\n\n"
       "// Solve (LU) x = b in place for the complex LU of kpp_decomp_cmplx_w, b given\n"
       "// in (XR, XI).\n"
       "template <class TJ, class TX>\n"
       "__device__ __noinline__ void kpp_solve_cmplx(const TJ& JR, const TJ& JI, TX& XR, TX& XI) {\n"
       "  for (int i = 0; i < KPP_NVAR; i++)\n"
       "    for (int j = kpp_lu_crow_c[i]; j < kpp_lu_diag_c[i]; j++) {\n"
       "      const int c = kpp_lu_icol_c[j];\n"
       "      XR[i] = XR[i] - (JR[j]*XR[c] - JI[j]*XI[c]);\n"
       "      XI[i] = XI[i] - (JR[j]*XI[c] + JI[j]*XR[c]);\n"
       "    }\n"
       "  for (int i = KPP_NVAR - 1; i >= 0; i--) {\n"
       "    const int d = kpp_lu_diag_c[i];\n"
       "    double sumr = XR[i], sumi = XI[i];\n"
       "    for (int j = d + 1; j < kpp_lu_crow_c[i + 1]; j++) {\n"
       "      const int c = kpp_lu_icol_c[j];\n"
       "      sumr = sumr - (JR[j]*XR[c] - JI[j]*XI[c]);\n"
       "      sumi = sumi - (JR[j]*XI[c] + JI[j]*XR[c]);\n"
       "    }\n"
       "    const double den = JR[d]*JR[d] + JI[d]*JI[d];\n"
       "    XR[i] = (sumr*JR[d] + sumi*JI[d])/den;\n"
       "    XI[i] = (sumi*JR[d] - sumr*JI[d])/den;\n"
       "  }\n"
       "}\n\n";
  } else {
    std::vector<std::vector<int>> pos(nvar, std::vector<int>(nvar, -1));
    for (int k = 0; k < m.lu_nonzero; k++) pos[m.lu_irow[k]][m.lu_icol[k]] = k;
    oc << "// In-place no-pivot sparse LU of the complex matrix (JR + i JI) of one cell;\n"
          "// returns k+1 when the real or the imaginary part of row k's diagonal entry\n"
          "// is zero on entry to its elimination, 0 on success.\n"
          "template <class TJ>\n"
          "__device__ KPP_MECH_INLINE int kpp_decomp_cmplx(TJ& JR, TJ& JI) {\n"
          "  double ar, ai, den;\n";
    for (int k = 0; k < nvar; k++) {
      const int dk = m.lu_diag[k];
      oc << "  if (JR[" << dk << "] == 0.0) return " << (k + 1) << ";\n"
         << "  if (JI[" << dk << "] == 0.0) return " << (k + 1) << ";\n";
      for (int kk = m.lu_crow[k]; kk < m.lu_diag[k]; kk++) {
        const int j = m.lu_icol[kk], dj = m.lu_diag[j];
        ops_decomp_c += 3 + 8;
        oc << "  den = JR[" << dj << "]*JR[" << dj << "] + JI[" << dj << "]*JI[" << dj << "];\n"
           << "  ar = -(JR[" << kk << "]*JR[" << dj << "] + JI[" << kk << "]*JI[" << dj
           << "])/den;\n"
           << "  ai = -(JI[" << kk << "]*JR[" << dj << "] - JR[" << kk << "]*JI[" << dj
           << "])/den;\n"
           << "  JR[" << kk << "] = -ar;\n  JI[" << kk << "] = -ai;\n";
        for (int jj = dj + 1; jj < m.lu_crow[j + 1]; jj++) {
          const int t = pos[k][m.lu_icol[jj]];
          ops_decomp_c += 8;
          oc << "  JR[" << t << "] = JR[" << t << "] + ar*JR[" << jj << "] - ai*JI[" << jj
             << "];\n"
             << "  JI[" << t << "] = JI[" << t << "] + ar*JI[" << jj << "] + ai*JR[" << jj
             << "];\n";
        }
      }
    }
    oc << "  (void)ar; (void)ai; (void)den;\n  return 0;\n}\n\n";

    oc << "// Solve (LU) x = b in place for the complex LU of kpp_decomp_cmplx, b given\n"
         "// in (XR, XI).\n"
         "template <class TJ, class TX>\n"
         "__device__ KPP_MECH_INLINE void kpp_solve_cmplx(const TJ& JR, const TJ& JI, TX& XR,"
         " TX& XI) {\n"
         "  double sumr, sumi, den;\n";
    for (int i = 0; i < nvar; i++)
      for (int j = m.lu_crow[i]; j < m.lu_diag[i]; j++) {
        const int c = m.lu_icol[j];
        ops_solve_c += 8;
        oc << "  XR[" << i << "] = XR[" << i << "] - (JR[" << j << "]*XR[" << c << "] - JI[" << j
          << "]*XI[" << c << "]);\n"
          << "  XI[" << i << "] = XI[" << i << "] - (JR[" << j << "]*XI[" << c << "] + JI[" << j
          << "]*XR[" << c << "]);\n";
      }
    for (int i = nvar - 1; i >= 0; i--) {
      const int d = m.lu_diag[i];
      oc << "  sumr = XR[" << i << "];\n  sumi = XI[" << i << "];\n";
      for (int j = d + 1; j < m.lu_crow[i + 1]; j++) {
        const int c = m.lu_icol[j];
        ops_solve_c += 8;
        oc << "  sumr = sumr - (JR[" << j << "]*XR[" << c << "] - JI[" << j << "]*XI[" << c
          << "]);\n"
          << "  sumi = sumi - (JR[" << j << "]*XI[" << c << "] + JI[" << j << "]*XR[" << c
          << "]);\n";
      }
      ops_solve_c += 11;
      oc << "  den = JR[" << d << "]*JR[" << d << "] + JI[" << d << "]*JI[" << d << "];\n"
        << "  XR[" << i << "] = (sumr*JR[" << d << "] + sumi*JI[" << d << "])/den;\n"
        << "  XI[" << i << "] = (sumi*JR[" << d << "] - sumr*JI[" << d << "])/den;\n";
    }
    oc << "  (void)sumr; (void)sumi; (void)den;\n}\n\n";
  }

  o << "// FP64 add/sub/mul/div operations per call of each function (for the\n"
       "// FP64 roofline; rate constants and the integrator's vector operations\n"
       "// are counted separately).\n"
    << "#define KPP_OPS_FUN " << ops_fun << "\n"
    << "#define KPP_OPS_JAC " << ops_jac << "\n"
    << "#define KPP_OPS_DECOMP " << ops_decomp << "\n"
    << "#define KPP_OPS_SOLVE " << ops_solve << "\n";
  oc << "#define KPP_OPS_DECOMP_CMPLX " << ops_decomp_c << "\n"
     << "#define KPP_OPS_SOLVE_CMPLX " << ops_solve_c << "\n";

  emit_coop_tables(o, m);

  std::ofstream f(out_prefix + ".cuh");
  if (!f) return false;
  f << o.str();
  if (!f) return false;
  // The complex LU lives in a header of its own, included after the main one
  // only by the integrators that need it (the Runge-Kutta methods).
  // ---- Jac_SP_Vec, JacTR_SP_Vec, KppSolveTR (src/gen.c:1763-1880,2036-2120):
  // the Jacobian (LU pattern) times a vector, its transpose times a vector,
  // and the transposed LU solve; the building blocks of the discrete
  // adjoint.  Terms are the Jacobian's structural entries (the diagonal
  // always counts), summed in the generator's order.
  std::ostringstream oa;
  {
    auto js = [&](int r, int c) { return r == c || m.jstruct[r][c]; };
    std::vector<std::vector<int>> pos(nvar, std::vector<int>(nvar, -1));
    for (int k = 0; k < m.lu_nonzero; k++) pos[m.lu_irow[k]][m.lu_icol[k]] = k;
    oa << "// Generated by kppcu: the Jacobian-vector products and the transposed LU\n"
          "// solve of the mechanism.  Include after the mechanism header.\n#pragma once\n\n"
          "// JUV = J UV, J in the LU pattern (JVS).\n"
          "template <class TJ, class TU, class TO>\n"
          "__device__ KPP_MECH_INLINE void kpp_jac_sp_vec(const TJ& JVS, const TU& UV, TO& JUV) {\n";
    for (int i = 0; i < nvar; i++) {
      P sum = cnst(0);
      for (int k = m.lu_crow[i]; k < m.lu_crow[i + 1]; k++)
        if (js(i, m.lu_icol[k]))
          sum = add(sum, mul(leaf("JVS[" + std::to_string(k) + "]"),
                             leaf("UV[" + std::to_string(m.lu_icol[k]) + "]")));
      oa << "  JUV[" << i << "] = " << print(sum) << ";\n";
    }
    oa << "}\n\n"
          "// JTUV = J^T UV, J in the LU pattern (JVS).\n"
          "template <class TJ, class TU, class TO>\n"
          "__device__ KPP_MECH_INLINE void kpp_jactr_sp_vec(const TJ& JVS, const TU& UV, TO& JTUV) {\n";
    for (int i = 0; i < nvar; i++) {
      P sum = cnst(0);
      for (int j = 0; j < nvar; j++)
        if (js(j, i))
          sum = add(sum, mul(leaf("JVS[" + std::to_string(pos[j][i]) + "]"),
                             leaf("UV[" + std::to_string(j) + "]")));
      oa << "  JTUV[" << i << "] = " << print(sum) << ";\n";
    }
    oa << "}\n\n"
          "// Solve (LU)^T XX = X for the factorised JVS.\n"
          "template <class TJ, class TX, class TY>\n"
          "__device__ KPP_MECH_INLINE void kpp_solve_tr(const TJ& JVS, const TX& X, TY& XX) {\n";
    // pos_t[c][r]: the LU entry (r, c), r != c, and the diagonal
    std::vector<std::vector<int>> pos_t(nvar, std::vector<int>(nvar, -1));
    for (int r = 0; r < nvar; r++) {
      for (int k = m.lu_crow[r]; k < m.lu_crow[r + 1]; k++)
        if (m.lu_icol[k] != r) pos_t[m.lu_icol[k]][r] = k;
      pos_t[r][r] = m.lu_diag[r];
    }
    for (int i = 0; i < nvar; i++) {
      P sum = leaf("X[" + std::to_string(i) + "]");
      for (int j = 0; j < i; j++)
        if (pos_t[i][j] >= 0)
          sum = sub(sum, mul(leaf("JVS[" + std::to_string(pos_t[i][j]) + "]"),
                             leaf("XX[" + std::to_string(j) + "]")));
      sum = divide(sum, leaf("JVS[" + std::to_string(m.lu_diag[i]) + "]"));
      oa << "  XX[" << i << "] = " << print(sum) << ";\n";
    }
    for (int i = nvar - 1; i >= 0; i--) {
      P sum = leaf("XX[" + std::to_string(i) + "]");
      bool any = false;
      for (int j = i + 1; j < nvar; j++)
        if (pos_t[i][j] >= 0) {
          sum = sub(sum, mul(leaf("JVS[" + std::to_string(pos_t[i][j]) + "]"),
                             leaf("XX[" + std::to_string(j) + "]")));
          any = true;
        }
      if (any) oa << "  XX[" << i << "] = " << print(sum) << ";\n";
    }
    oa << "}\n";
  }
  {
    std::ofstream fa(out_prefix + "_adj.cuh");
    if (!fa) return false;
    fa << oa.str();
    if (!fa) return false;
  }

  std::ofstream fc(out_prefix + "_cmplx.cuh");
  if (!fc) return false;
  fc << "// Generated by kppcu: complex sparse LU of the mechanism (util/sutil.c:28-90),\n"
        "// unrolled.  Include after the mechanism header.\n#pragma once\n\n"
     << oc.str();
  return (bool)fc;
}

}  // namespace kppcu
