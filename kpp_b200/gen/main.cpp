// kppcu: compile a KPP mechanism into CUDA device code for the batched
// Rosenbrock engine.
//
//   kppcu <mechanism.kpp> -o <out_prefix> [--home <KPP_HOME>] [--root <name>]
//
// Writes <out_prefix>.cuh (device code + tables, see emit_cuda.cpp) and
// <out_prefix>.json (species order, sparsity pattern and reaction kinds, for
// tools and tests).  The role is that of the reference generator's C
// emitter (src/code_c.c selected from src/gen.c:3905-3916) for the new
// `#LANGUAGE CUDA` target.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>

#include "mechanism.hpp"

using namespace kppcu;

static std::string json_str(const std::string& s) {
  std::string o = "\"";
  for (char c : s) {
    if (c == '"' || c == '\\') o += '\\';
    if (c == '\n') { o += "\\n"; continue; }
    o += c;
  }
  return o + "\"";
}

static void json_ints(std::ofstream& f, const char* key, const std::vector<int>& v, bool last = false) {
  f << "  \"" << key << "\": [";
  for (size_t i = 0; i < v.size(); i++) f << (i ? ", " : "") << v[i];
  f << "]" << (last ? "\n" : ",\n");
}

static bool write_json(const Mechanism& m, const std::string& path) {
  std::ofstream f(path);
  if (!f) return false;
  f << "{\n";
  f << "  \"root\": " << json_str(m.root) << ",\n";
  f << "  \"nvar\": " << m.nvar << ", \"nfix\": " << m.nfix << ", \"nspec\": " << m.nspec
    << ", \"nvaract\": " << m.nvaract << ", \"nreact\": " << m.nreact()
    << ", \"nonzero\": " << m.nonzero << ", \"lu_nonzero\": " << m.lu_nonzero << ",\n";
  char buf[64];
  std::snprintf(buf, sizeof buf, "%.17g", m.cfactor);
  f << "  \"cfactor\": " << buf << ",\n";
  f << "  \"species\": [";
  for (int i = 0; i < m.nspec; i++)
    f << (i ? ", " : "") << json_str(m.table[m.order[m.spc_slot[i]]].name);
  f << "],\n";
  std::vector<int> kinds;
  for (const Reaction& r : m.reactions) kinds.push_back((int)r.kind);
  json_ints(f, "rate_kind", kinds);
  f << "  \"rates\": [";
  for (int j = 0; j < m.nreact(); j++) f << (j ? ", " : "") << json_str(m.reactions[j].rate);
  f << "],\n";
  json_ints(f, "lu_irow", m.lu_irow);
  json_ints(f, "lu_icol", m.lu_icol);
  json_ints(f, "lu_crow", m.lu_crow);
  json_ints(f, "lu_diag", m.lu_diag, true);
  f << "}\n";
  return (bool)f;
}

int main(int argc, char** argv) {
  std::string in, out, home, root;
  if (const char* h = std::getenv("KPP_HOME")) home = h;
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    if (a == "-o" && i + 1 < argc) out = argv[++i];
    else if (a == "--home" && i + 1 < argc) home = argv[++i];
    else if (a == "--root" && i + 1 < argc) root = argv[++i];
    else if (!a.empty() && a[0] != '-') in = a;
    else {
      std::fprintf(stderr, "kppcu: unknown argument %s\n", a.c_str());
      return 1;
    }
  }
  if (in.empty() || out.empty()) {
    std::fprintf(stderr, "usage: kppcu <mechanism.kpp> -o <out_prefix> [--home KPP_HOME] [--root name]\n");
    return 1;
  }
  Mechanism m;
  if (root.empty()) {
    size_t s = in.rfind('/');
    root = in.substr(s == std::string::npos ? 0 : s + 1);
    size_t d = root.rfind('.');
    if (d != std::string::npos) root = root.substr(0, d);
  }
  m.root = root;
  if (!parse_mechanism(in, home, m)) {
    std::fprintf(stderr, "kppcu: %d errors in %s\n", m.errors, in.c_str());
    return 2;
  }
  for (const std::string& w : m.warnings) std::fprintf(stderr, "kppcu: warning: %s\n", w.c_str());
  if (m.reactions.empty()) {
    std::fprintf(stderr, "kppcu: no equations in %s\n", in.c_str());
    return 2;
  }
  build_structure(m);
  if (m.nvar == 0) {
    std::fprintf(stderr, "kppcu: no variable species\n");
    return 2;
  }
  if (!emit_cuda(m, out) || !emit_host(m, out) || !write_json(m, out + ".json")) {
    std::fprintf(stderr, "kppcu: cannot write %s\n", out.c_str());
    return 3;
  }
  std::printf("kppcu: %s: NVAR=%d NFIX=%d NREACT=%d LU_NONZERO=%d -> %s.cuh\n", m.root.c_str(),
              m.nvar, m.nfix, m.nreact(), m.lu_nonzero, out.c_str());
  return 0;
}
