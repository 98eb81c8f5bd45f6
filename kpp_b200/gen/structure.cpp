// kppcu structure pass: species order and sparsity of the Jacobian and of its
// LU factors.
//
// The order of the variable species fixes the sparsity pattern of the LU
// factors, and with it every line of the generated Jacobian, LU and solve
// code.  It therefore follows the reference generator's rules exactly:
//   1. variables sorted reactive-first, then by declaration order; fixed
//      species by declaration order; dummy species dropped
//      (ReorderSpecies(UNSORT), src/kpp.c:273-403, comparator CodeRCmp :66-80);
//   2. a Markowitz pivot order: at each elimination step take the first row i
//      with the smallest (row count - 1) * (column count - 1) over the active
//      submatrix, swap it into place, and add its pattern into the rows below
//      (BestSparsity, src/kpp.c:220-271), then reorder by that pivot sequence;
//   3. the Jacobian pattern J[i][j] = (i == j) or some equation with a nonzero
//      net coefficient for i consumes j (UpdateStructJ, src/kpp.c:113-131) and
//      its symbolic LU fill (ComputeLUStructJ, src/kpp.c:133-158);
//   4. row-major compressed storage with the diagonal always present
//      (NonZero, src/gen.c:331-356).
#include <algorithm>

#include "mechanism.hpp"

namespace kppcu {

namespace {

// J pattern over the first nvar entries of `ord` (slots).
std::vector<std::vector<int>> jacobian_pattern(const Mechanism& m, const std::vector<int>& ord,
                                               int nvar) {
  std::vector<std::vector<int>> j(nvar, std::vector<int>(nvar, 0));
  int nr = m.nreact();
  for (int a = 0; a < nvar; a++) {
    j[a][a] = 1;
    const std::vector<float>& net = m.net[ord[a]];
    for (int b = 0; b < nvar; b++) {
      const std::vector<float>& lb = m.left[ord[b]];
      for (int k = 0; k < nr; k++)
        if (net[k] * (lb[k] != 0.0f ? 1.0f : 0.0f) != 0.0f) { j[a][b] = 1; break; }
    }
  }
  return j;
}

}  // namespace

void build_structure(Mechanism& m) {
  // ---- 1. variables reactive-first, then by code; fixed by code
  std::vector<int> vars, fixes;
  for (size_t s = 0; s < m.order.size(); s++) {
    int code = m.order[s];
    int type = code < (int)m.table.size() ? m.table[code].type : SPC_DUMMY;
    if (type == SPC_VAR) vars.push_back((int)s);
    else if (type == SPC_FIX) fixes.push_back((int)s);
  }
  std::sort(vars.begin(), vars.end(), [&](int a, int b) {
    if (m.reactive[a] != m.reactive[b]) return m.reactive[a] > m.reactive[b];
    return m.order[a] < m.order[b];
  });
  std::sort(fixes.begin(), fixes.end(), [&](int a, int b) { return m.order[a] < m.order[b]; });
  int nvar = (int)vars.size();

  // ---- 2. Markowitz pivot sequence over the unsorted variable order
  if (m.reorder && nvar > 0) {
    std::vector<std::vector<int>> lu = jacobian_pattern(m, vars, nvar);
    std::vector<int> seq = vars;
    for (int s = 0; s < nvar - 1; s++) {
      long best = -1;
      int best_i = 0;
      for (int i = s; i < nvar; i++) {
        long rows = 0, cols = 0;
        for (int k = s; k < nvar; k++) {
          rows += lu[i][k] ? 1 : 0;
          cols += lu[k][i] ? 1 : 0;
        }
        long cost = (rows - 1) * (cols - 1);
        if (best < 0 || cost < best) { best = cost; best_i = i; }
      }
      std::swap(lu[s], lu[best_i]);
      for (int i = 0; i < nvar; i++) std::swap(lu[i][s], lu[i][best_i]);
      std::swap(seq[s], seq[best_i]);
      for (int i = s + 1; i < nvar; i++)
        if (lu[i][s])
          for (int k = s; k < nvar; k++) lu[i][k] += lu[s][k];
    }
    vars = seq;
  }

  m.spc_slot = vars;
  m.spc_slot.insert(m.spc_slot.end(), fixes.begin(), fixes.end());
  m.nvar = nvar;
  m.nfix = (int)fixes.size();
  m.nspec = m.nvar + m.nfix;
  m.nvaract = 0;
  for (int v : vars) m.nvaract += m.reactive[v] ? 1 : 0;

  // ---- 3. Jacobian pattern and its LU fill in the final order
  std::vector<std::vector<int>> j = jacobian_pattern(m, vars, nvar);
  std::vector<std::vector<int>> lu = j;
  for (int c = 0; c < nvar - 1; c++)
    for (int i = c + 1; i < nvar; i++)
      if (lu[i][c])
        for (int k = c; k < nvar; k++)
          if (lu[c][k]) lu[i][k] = 1;
  m.jstruct.assign(nvar, std::vector<char>(nvar, 0));
  m.lustruct.assign(nvar, std::vector<char>(nvar, 0));
  for (int a = 0; a < nvar; a++)
    for (int b = 0; b < nvar; b++) {
      m.jstruct[a][b] = j[a][b] != 0;
      m.lustruct[a][b] = lu[a][b] != 0;
    }

  // ---- 4. compressed row storage, diagonal always stored
  m.nonzero = 0;
  for (int a = 0; a < nvar; a++)
    for (int b = 0; b < nvar; b++) m.nonzero += (a == b || m.jstruct[a][b]) ? 1 : 0;
  m.lu_irow.clear();
  m.lu_icol.clear();
  m.lu_crow.assign(nvar + 1, 0);
  m.lu_diag.assign(nvar + 1, 0);
  for (int a = 0; a < nvar; a++) {
    m.lu_crow[a] = (int)m.lu_icol.size();
    for (int b = 0; b < nvar; b++) {
      if (a == b || m.lustruct[a][b]) {
        m.lu_irow.push_back(a);
        m.lu_icol.push_back(b);
      }
      if (a == b) m.lu_diag[a] = (int)m.lu_icol.size() - 1;
    }
  }
  m.lu_nonzero = (int)m.lu_icol.size();
  m.lu_crow[nvar] = m.lu_nonzero;
  m.lu_diag[nvar] = m.lu_nonzero;
}

}  // namespace kppcu
