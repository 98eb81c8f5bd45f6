// kppcu front end: the KPP mechanism language.
//
// The language is defined by the reference's scanner and grammar
// (src/scan.l:37-298 for tokens and scanner modes, src/scan.l:301-341 for the
// command keywords, src/scan.y:105-372 for the grammar) and by the semantic
// actions in src/scanner.c (DeclareSpecies :506, SetSpcType :522,
// AssignInitialValue :556, StoreEquationRate :604-628, ProcessTerm :712-766,
// ParseEquationFile :873-920).  This is an independent implementation of
// those rules: a mode-driven scanner with longest-match token selection and a
// statement parser that updates a kppcu::Mechanism directly.
//
// Facts that decide the generated arithmetic and are therefore kept exactly:
//   * species codes are declaration order, with a dummy species at code 0
//     (src/scanner.c:907-913); equations list species in first-appearance
//     order (the reference's Code[] array);
//   * stoichiometric coefficients accumulate in single precision;
//   * a rate is the concatenation of the whitespace-separated pieces between
//     ':' and ';' (comments removed); a rate that is a bare number becomes a
//     single-precision constant, anything else an expression, and every
//     equation with `hv` a photolysis expression.
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

#include "mechanism.hpp"

namespace kppcu {

static const int CODE_HV = 1 << 20;
static const int CODE_PROD = (1 << 20) + 1;

static bool eq_nocase(const std::string& a, const std::string& b) {
  if (a.size() != b.size()) return false;
  for (size_t i = 0; i < a.size(); i++)
    if (std::toupper((unsigned char)a[i]) != std::toupper((unsigned char)b[i])) return false;
  return true;
}

int Mechanism::find_species(const std::string& name) const {
  for (size_t i = 0; i < table.size(); i++)
    if (eq_nocase(table[i].name, name)) return (int)i;
  if (eq_nocase(name, "HV")) return CODE_HV;
  if (eq_nocase(name, "PROD")) return CODE_PROD;
  return -1;
}

int Mechanism::slot_for(int code) {
  auto it = slot_of_code.find(code);
  if (it != slot_of_code.end()) return it->second;
  int s = (int)order.size();
  order.push_back(code);
  slot_of_code[code] = s;
  reactive.push_back(0);
  left.emplace_back();
  right.emplace_back();
  net.emplace_back();
  return s;
}

// ---------------------------------------------------------------------------
// Scanner
// ---------------------------------------------------------------------------
namespace {

enum Mode {
  M_TOP, M_CMD, M_PARAM, M_INC, M_MODEL, M_INTEG, M_IGNORE, M_ATOMS, M_SPECIES,
  M_SETSPC, M_INIT, M_EQN, M_EQNTAG, M_RATE, M_FAMILY, M_LIST, M_INLCTX, M_INLCODE
};

enum TokKind {
  T_END, T_CMD, T_PARAM, T_ID, T_NUM, T_EQ, T_PLUS, T_SIGN, T_SEMI, T_COLON, T_LT,
  T_GT, T_TAG, T_COEF, T_RATE, T_INLCTX, T_INLTEXT, T_INLEND
};

struct Token {
  TokKind kind = T_END;
  std::string text;
  std::string cmd;  // upper-case command name for T_CMD
  int line = 0;
};

struct Source {
  std::string text;
  size_t pos = 0;
  std::string name;
  int line = 1;
};

// command keyword -> mode that follows it; emits a token unless `silent`
struct Keyword {
  const char* name;
  Mode next;
  bool silent;
};

const Keyword kKeywords[] = {
    {"INCLUDE", M_INC, true},      {"MODEL", M_MODEL, true},
    {"INTEGRATOR", M_INTEG, true}, {"JACOBIAN", M_PARAM, false},
    {"HESSIAN", M_PARAM, false},   {"DECLARE", M_PARAM, false},
    {"STOICMAT", M_PARAM, false},  {"STOCHASTIC", M_PARAM, false},
    {"DOUBLE", M_PARAM, false},    {"REORDER", M_PARAM, false},
    {"MEX", M_PARAM, false},       {"DUMMYINDEX", M_PARAM, false},
    {"EQNTAGS", M_PARAM, false},   {"FUNCTION", M_PARAM, false},
    {"ATOMS", M_ATOMS, false},     {"CHECK", M_ATOMS, false},
    {"CHECKALL", M_TOP, false},    {"DEFVAR", M_SPECIES, false},
    {"DEFFIX", M_SPECIES, false},  {"SETVAR", M_SETSPC, false},
    {"SETFIX", M_SETSPC, false},   {"INITVALUES", M_INIT, false},
    {"EQUATIONS", M_EQN, false},   {"FAMILIES", M_FAMILY, false},
    {"LOOKAT", M_LIST, false},     {"LOOKATALL", M_TOP, false},
    {"MONITOR", M_LIST, false},    {"WRITE_ATM", M_TOP, false},
    {"WRITE_SPC", M_TOP, false},   {"WRITE_MAT", M_TOP, false},
    {"LANGUAGE", M_PARAM, false},  {"INLINE", M_INLCTX, false},
    {"ENDINLINE", M_TOP, false},   {"INTFILE", M_PARAM, false},
    {"DRIVER", M_PARAM, false},    {"FLUX", M_PARAM, false},
    {"UPPERCASEF90", M_PARAM, false}, {"MINVERSION", M_PARAM, false},
    {"AUTOREDUCE", M_PARAM, false},   {"GRAPH", M_PARAM, false},
};

bool is_lit(char c) { return std::isalpha((unsigned char)c) || c == '_'; }
bool is_word(char c) { return std::isalnum((unsigned char)c) || c == '_'; }
bool is_digit(char c) { return std::isdigit((unsigned char)c) != 0; }

class Scanner {
 public:
  Scanner(Mechanism& m, std::string home, std::string top_dir)
      : m_(m), home_(std::move(home)), top_dir_(std::move(top_dir)) {}

  bool open(const std::string& path) { return push_file(path); }
  std::string where() const {
    if (src_.empty()) return "<eof>";
    return src_.back().name + ":" + std::to_string(src_.back().line);
  }
  void error(const std::string& msg) {
    std::fprintf(stderr, "kppcu: error: %s: %s\n", where().c_str(), msg.c_str());
    m_.errors++;
  }
  void warning(const std::string& msg) {
    m_.warnings.push_back(where() + ": " + msg);
  }

  Token next();

 private:
  Mechanism& m_;
  std::string home_, top_dir_;
  std::vector<Source> src_;
  Mode mode_ = M_TOP;

  bool push_file(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    std::stringstream ss;
    ss << f.rdbuf();
    Source s;
    s.text = ss.str();
    s.name = path;
    src_.push_back(std::move(s));
    return true;
  }

  static bool file_exists(const std::string& p) {
    std::ifstream f(p);
    return (bool)f;
  }

  // File lookup: name (adding `ext` when it has none) as given, then next to
  // the top-level file, then under $KPP_HOME/<dir>.
  std::string locate(const std::string& name, const std::string& dir, const std::string& ext) {
    std::string n = name;
    size_t slash = n.rfind('/');
    size_t dot = n.rfind('.');
    if (dot == std::string::npos || (slash != std::string::npos && dot < slash)) n += ext;
    if (file_exists(n)) return n;
    if (!top_dir_.empty() && n[0] != '/' && file_exists(top_dir_ + "/" + n)) return top_dir_ + "/" + n;
    if (!home_.empty() && file_exists(home_ + "/" + dir + "/" + n)) return home_ + "/" + dir + "/" + n;
    return n;
  }

  void include(const std::string& name, const std::string& dir, const std::string& ext) {
    std::string p = locate(name, dir, ext);
    if (src_.size() > 10) {
      warning("include nested too deep: " + name);
      return;
    }
    if (!push_file(p)) {
      error("cannot read file " + p);
      std::exit(3);
    }
  }

  // Length of the longest match of the token classes used below.
  static size_t len_while(const std::string& t, size_t p, bool (*ok)(char)) {
    size_t i = p;
    while (i < t.size() && ok(t[i])) i++;
    return i - p;
  }
  static bool string_char(char c) { return !std::strchr(" \t\n{}#;", c) && c != 0; }
  static size_t len_string(const std::string& t, size_t p) { return len_while(t, p, string_char); }
  static size_t len_id(const std::string& t, size_t p) {
    if (p >= t.size() || !is_lit(t[p])) return 0;
    return len_while(t, p, is_word);
  }
  static size_t len_digits(const std::string& t, size_t p) { return len_while(t, p, is_digit); }
  static size_t len_signed_digits(const std::string& t, size_t p) {
    size_t i = p;
    if (i < t.size() && (t[i] == '+' || t[i] == '-')) i++;
    size_t d = len_digits(t, i);
    return d ? (i - p) + d : 0;
  }
  static size_t len_exponent(const std::string& t, size_t p) {
    if (p >= t.size() || !std::strchr("eEdD", t[p]) || t[p] == 0) return 0;
    size_t e = len_signed_digits(t, p + 1);
    return e ? 1 + e : 0;
  }
  // [+-]?digits? '.'? digits? exponent?   (signed = initial-value numbers)
  static size_t len_number(const std::string& t, size_t p, bool allow_sign) {
    size_t i = p;
    if (allow_sign) i += len_signed_digits(t, i);
    else i += len_digits(t, i);
    if (i < t.size() && t[i] == '.') i++;
    i += len_digits(t, i);
    return (i - p) + len_exponent(t, i);
  }

  Token make(TokKind k, const std::string& text) {
    Token tk;
    tk.kind = k;
    tk.text = text;
    tk.line = src_.empty() ? 0 : src_.back().line;
    return tk;
  }
};

Token Scanner::next() {
  for (;;) {
    if (src_.empty()) return make(T_END, "");
    Source& s = src_.back();
    const std::string& t = s.text;
    if (s.pos >= t.size()) {
      if (src_.size() > 1) {
        src_.pop_back();
        continue;
      }
      src_.clear();
      return make(T_END, "");
    }
    size_t p = s.pos;
    char c = t[p];

    if (mode_ == M_INLCODE) {
      if (c == '#') {
        size_t i = p + 1;
        while (i < t.size() && t[i] != ' ' && t[i] != '\t' && t[i] != '\n') i++;
        std::string word = t.substr(p, i - p);
        s.pos = i;
        if (eq_nocase(word.substr(1), "ENDINLINE")) {
          mode_ = M_TOP;
          return make(T_INLEND, word);
        }
        return make(T_INLTEXT, word);
      }
      if (c == '\n') {
        s.pos++;
        s.line++;
        return make(T_INLTEXT, "\n");
      }
      size_t i = p;
      while (i < t.size() && t[i] != '#' && t[i] != '\n') i++;
      s.pos = i;
      return make(T_INLTEXT, t.substr(p, i - p));
    }

    // Rules shared by every other mode: blanks, newlines, comments, commands.
    if (c == ' ' || c == '\t' || c == '\r') {
      s.pos++;
      continue;
    }
    if (c == '\n') {
      s.pos++;
      s.line++;
      continue;
    }
    if (c == '{') {
      size_t i = p + 1;
      while (i < t.size() && t[i] != '}') {
        if (t[i] == '\n') s.line++;
        i++;
      }
      s.pos = (i < t.size()) ? i + 1 : i;
      continue;
    }
    bool string_mode = (mode_ == M_CMD || mode_ == M_PARAM || mode_ == M_INC || mode_ == M_MODEL ||
                        mode_ == M_INTEG || mode_ == M_IGNORE || mode_ == M_RATE ||
                        mode_ == M_INLCTX);
    if (c == '/' && p + 1 < t.size() && t[p + 1] == '/') {
      // A token of a string mode that is longer than "//" wins (longest match).
      if (!(string_mode && len_string(t, p) > 2)) {
        size_t i = p;
        while (i < t.size() && t[i] != '\n') i++;
        s.pos = i;
        continue;
      }
    }
    if (c == '#') {
      s.pos++;
      mode_ = M_CMD;
      continue;
    }

    switch (mode_) {
      case M_CMD: {
        size_t n = len_string(t, p);
        std::string word = t.substr(p, n);
        s.pos += n;
        const Keyword* kw = nullptr;
        for (const Keyword& k : kKeywords)
          if (eq_nocase(word, k.name)) kw = &k;
        if (!kw) {
          error("'" + word + "': Unknown command (ignored)");
          mode_ = M_IGNORE;
          continue;
        }
        mode_ = kw->next;
        if (kw->silent) {
          // INCLUDE / MODEL / INTEGRATOR take their argument in the next mode
          continue;
        }
        Token tk = make(T_CMD, word);
        tk.cmd = kw->name;
        return tk;
      }
      case M_INC: case M_MODEL: case M_INTEG: {
        size_t n = len_string(t, p);
        std::string arg = t.substr(p, n);
        s.pos += n;
        Mode was = mode_;
        mode_ = M_IGNORE;
        if (was == M_INC) include(arg, "models", "");
        else if (was == M_MODEL) include(arg, "models", ".def");
        else {
          m_.integrator = arg;
          include(arg, "int", ".def");
        }
        continue;
      }
      case M_PARAM: {
        size_t n = len_string(t, p);
        s.pos += n;
        mode_ = M_IGNORE;
        return make(T_PARAM, t.substr(p, n));
      }
      case M_IGNORE: {
        size_t n = len_string(t, p);
        if (n == 0) n = 1;
        error("Extra parameter on command line '" + t.substr(p, n) + "'");
        s.pos += n;
        continue;
      }
      case M_INLCTX: {
        size_t n = len_string(t, p);
        if (n == 0) { s.pos++; continue; }
        s.pos += n;
        mode_ = M_INLCODE;
        return make(T_INLCTX, t.substr(p, n));
      }
      case M_ATOMS: case M_LIST: case M_SETSPC: {
        size_t n = len_id(t, p);
        if (n) { s.pos += n; return make(T_ID, t.substr(p, n)); }
        if (c == ';') { s.pos++; return make(T_SEMI, ";"); }
        s.pos++;  // characters without a rule are skipped
        continue;
      }
      case M_SPECIES: case M_FAMILY: {
        size_t n = len_id(t, p);
        if (n) { s.pos += n; return make(T_ID, t.substr(p, n)); }
        n = len_digits(t, p);
        if (n) { s.pos += n; return make(T_NUM, t.substr(p, n)); }
        s.pos++;
        if (c == '=') return make(T_EQ, "=");
        if (c == '+') return make(T_PLUS, "+");
        if (c == ';') return make(T_SEMI, ";");
        if (c == ':' && mode_ == M_FAMILY) return make(T_COLON, ":");
        error(std::string("Invalid character '") + c + "' in species definition");
        continue;
      }
      case M_INIT: {
        size_t ni = len_id(t, p), nf = len_number(t, p, true);
        if (ni && ni >= nf) { s.pos += ni; return make(T_ID, t.substr(p, ni)); }
        if (c == '=') { s.pos++; return make(T_EQ, "="); }
        if (c == ';') { s.pos++; return make(T_SEMI, ";"); }
        if (nf) { s.pos += nf; return make(T_NUM, t.substr(p, nf)); }
        s.pos++;
        if (c != '=' && c != ';') error(std::string("Invalid character '") + c + "' in initial values");
        continue;
      }
      case M_EQN: {
        size_t ni = len_id(t, p);
        size_t ns = (ni && p + ni < t.size() && t[p + ni] == '*') ? ni + 1 : 0;
        size_t nu = len_number(t, p, false);
        // longest match; on a tie the species-with-'*' rule, then identifiers,
        // win over numbers
        if (ns && ns >= ni && ns >= nu) { s.pos += ns; return make(T_COEF, t.substr(p, ns)); }
        if (ni && ni >= nu) { s.pos += ni; return make(T_ID, t.substr(p, ni)); }
        if (c == '=' ) { s.pos++; return make(T_EQ, "="); }
        if (nu) { s.pos += nu; return make(T_COEF, t.substr(p, nu)); }
        s.pos++;
        if (c == ':') { mode_ = M_RATE; return make(T_COLON, ":"); }
        if (c == '+' || c == '-') return make(T_SIGN, std::string(1, c));
        if (c == '<') { mode_ = M_EQNTAG; return make(T_LT, "<"); }
        continue;
      }
      case M_EQNTAG: {
        size_t n = len_while(t, p, is_word);
        if (n) { s.pos += n; return make(T_TAG, t.substr(p, n)); }
        s.pos++;
        if (c == '>') { mode_ = M_EQN; return make(T_GT, ">"); }
        continue;
      }
      case M_RATE: {
        if (c == ';') { s.pos++; mode_ = M_EQN; return make(T_SEMI, ";"); }
        size_t n = len_string(t, p);
        if (n) { s.pos += n; return make(T_RATE, t.substr(p, n)); }
        s.pos++;
        continue;
      }
      case M_TOP: default:
        s.pos++;  // text outside any command is ignored
        continue;
    }
  }
}

// ---------------------------------------------------------------------------
// Parser
// ---------------------------------------------------------------------------
class Parser {
 public:
  Parser(Mechanism& m, Scanner& sc) : m_(m), sc_(sc) {}
  void run();

 private:
  Mechanism& m_;
  Scanner& sc_;
  Token look_;
  bool have_ = false;
  std::string section_;
  bool photo_ = false;

  Token& peek() {
    if (!have_) { look_ = sc_.next(); have_ = true; }
    return look_;
  }
  Token take() { Token t = peek(); have_ = false; return t; }
  bool at(TokKind k) { return peek().kind == k; }
  void skip_semicolons() {
    if (!at(T_SEMI)) { sc_.error("missing ';'"); return; }
    take();
    while (at(T_SEMI)) take();
  }
  void recover() {
    sc_.error("syntax error near '" + peek().text + "'");
    while (!at(T_END) && !at(T_CMD) && !at(T_SEMI)) take();
    if (at(T_SEMI)) skip_semicolons();
  }

  void command(const Token& t);
  void param_command(const std::string& cmd, const std::string& arg);
  void species_list(int type);
  void init_list();
  void equation_list();
  void equation();
  void term_list(int side);
  void process_term(int side, const std::string& sign, const std::string& coef,
                    const std::string& name);
  void store_rate(const std::string& rate, const std::string& tag);
  void declare_species(int type, const std::string& name);
  void set_type(int type, const std::string& name);
  void assign_initial(const std::string& name, const std::string& value);
  void inline_block();
};

void Parser::run() {
  // The dummy species "???" occupies code 0 (src/scanner.c:911).
  Species dummy;
  dummy.name = "???";
  dummy.type = SPC_DUMMY;
  m_.table.push_back(dummy);
  while (!at(T_END)) {
    Token t = take();
    if (t.kind != T_CMD) {
      sc_.error("unexpected '" + t.text + "'");
      continue;
    }
    command(t);
  }
}

void Parser::command(const Token& t) {
  const std::string& c = t.cmd;
  section_ = c;
  if (c == "ATOMS" || c == "CHECK" || c == "LOOKAT" || c == "MONITOR") {
    while (at(T_ID)) { take(); skip_semicolons(); }
    return;
  }
  if (c == "SETVAR" || c == "SETFIX") {
    while (at(T_ID)) {
      set_type(c == "SETVAR" ? SPC_VAR : SPC_FIX, take().text);
      skip_semicolons();
    }
    return;
  }
  if (c == "DEFVAR" || c == "DEFFIX") { species_list(c == "DEFVAR" ? SPC_VAR : SPC_FIX); return; }
  if (c == "INITVALUES") { init_list(); return; }
  if (c == "EQUATIONS") { equation_list(); return; }
  if (c == "FAMILIES") {
    sc_.warning("#FAMILIES is not used by the CUDA path and is ignored");
    while (at(T_ID) || at(T_NUM) || at(T_COLON) || at(T_PLUS) || at(T_SEMI)) take();
    return;
  }
  if (c == "CHECKALL" || c == "LOOKATALL" || c == "WRITE_ATM" || c == "WRITE_SPC" ||
      c == "WRITE_MAT" || c == "ENDINLINE")
    return;
  if (c == "INLINE") { inline_block(); return; }
  if (!at(T_PARAM)) { sc_.error("#" + c + " needs a parameter"); return; }
  param_command(c, take().text);
}

static bool on_off(const std::string& v, bool* out) {
  if (eq_nocase(v, "ON")) { *out = true; return true; }
  if (eq_nocase(v, "OFF")) { *out = false; return true; }
  return false;
}

void Parser::param_command(const std::string& c, const std::string& arg) {
  bool b = false;
  if (c == "LANGUAGE") {
    m_.language = arg;
    if (!eq_nocase(arg, "CUDA"))
      sc_.warning("#LANGUAGE " + arg + ": kppcu writes CUDA; the " + arg +
                  " inline blocks are ignored and the CUDA_* blocks are used");
  } else if (c == "INTFILE") {
    m_.integrator = arg;
  } else if (c == "REORDER") {
    if (!on_off(arg, &m_.reorder)) sc_.error("#REORDER [ON|OFF]");
  } else if (c == "DOUBLE") {
    if (!on_off(arg, &m_.use_double)) sc_.error("#DOUBLE [ON|OFF]");
    if (!m_.use_double) sc_.warning("#DOUBLE OFF: the CUDA Rosenbrock path always computes in FP64");
  } else if (c == "EQNTAGS") {
    if (!on_off(arg, &m_.eqntags)) sc_.error("#EQNTAGS [ON|OFF]");
  } else if (c == "JACOBIAN") {
    if (!eq_nocase(arg, "SPARSE_LU_ROW"))
      sc_.warning("#JACOBIAN " + arg + ": the CUDA path always uses SPARSE_LU_ROW");
  } else if (c == "FLUX" || c == "AUTOREDUCE" || c == "STOCHASTIC") {
    if (on_off(arg, &b) && b) sc_.error("#" + c + " ON is not supported by the CUDA path");
  } else {
    // HESSIAN, STOICMAT, MEX, DECLARE, DUMMYINDEX, FUNCTION, DRIVER,
    // UPPERCASEF90, MINVERSION, GRAPH: no effect on the CUDA path.
  }
}

void Parser::declare_species(int type, const std::string& name) {
  if (m_.find_species(name) >= 0 && m_.find_species(name) < (int)m_.table.size()) {
    sc_.error("Multiple declaration for species " + name);
    return;
  }
  Species s;
  s.name = name;
  s.type = type;
  m_.table.push_back(s);
}

void Parser::species_list(int type) {
  while (at(T_ID)) {
    std::string name = take().text;
    if (at(T_EQ)) {  // atom composition: [n]ATOM (+ [n]ATOM)*
      take();
      for (;;) {
        if (at(T_NUM)) take();
        if (!at(T_ID)) { sc_.error("missing atom after '" + name + "'"); break; }
        take();
        if (!at(T_PLUS)) break;
        take();
      }
    }
    declare_species(type, name);
    if (at(T_SEMI)) skip_semicolons();
    else recover();
  }
}

void Parser::set_type(int type, const std::string& name) {
  auto retype = [&](int from) {
    for (Species& s : m_.table)
      if (from < 0 || s.type == from) s.type = type;
  };
  if (eq_nocase(name, "VAR_SPEC")) { retype(SPC_VAR); return; }
  if (eq_nocase(name, "FIX_SPEC")) { retype(SPC_FIX); return; }
  if (eq_nocase(name, "ALL_SPEC")) { retype(-1); return; }
  int code = m_.find_species(name);
  if (code < 0 || code >= (int)m_.table.size()) { sc_.error("Undefined species " + name); return; }
  m_.table[code].type = type;
}

void Parser::assign_initial(const std::string& name, const std::string& value) {
  if (eq_nocase(name, "CFACTOR")) {
    char* end = nullptr;
    double v = std::strtod(value.c_str(), &end);
    if (end == value.c_str()) { sc_.warning("Invalid CFACTOR value: " + value); return; }
    m_.cfactor = v;
    return;
  }
  if (eq_nocase(name, "VAR_SPEC")) { m_.var_default = value; return; }
  if (eq_nocase(name, "FIX_SPEC")) { m_.fix_default = value; return; }
  if (eq_nocase(name, "ALL_SPEC")) { m_.var_default = value; m_.fix_default = value; return; }
  int code = m_.find_species(name);
  if (code < 0 || code >= (int)m_.table.size()) { sc_.error("Undefined species " + name); return; }
  m_.table[code].ival = value;
}

void Parser::init_list() {
  while (at(T_ID)) {
    std::string name = take().text;
    if (!at(T_EQ)) { recover(); continue; }
    take();
    if (!at(T_NUM)) { recover(); continue; }
    assign_initial(name, take().text);
    if (at(T_SEMI)) skip_semicolons();
    else recover();
  }
}

void Parser::process_term(int side, const std::string& sign, const std::string& coef,
                          const std::string& name) {
  int code = m_.find_species(name);
  if (code < 0) { sc_.error("Undefined species " + name); return; }
  if (code == CODE_HV) photo_ = true;
  int slot = m_.slot_for(code);
  std::string num = sign + coef;
  char* end = nullptr;
  double val = std::strtod(num.c_str(), &end);
  if (end == num.c_str()) { sc_.error("invalid coefficient '" + coef + "'"); return; }
  int eq = (int)m_.reactions.size();
  for (auto* v : {&m_.left[slot], &m_.right[slot], &m_.net[slot]})
    if ((int)v->size() <= eq) v->resize(eq + 1, 0.0f);
  // single-precision accumulation, as in the reference's float matrices
  if (side == 0) {
    m_.left[slot][eq] = (float)((double)m_.left[slot][eq] + val);
    m_.net[slot][eq] = (float)((double)m_.net[slot][eq] - val);
    m_.reactive[slot] = 1;
  } else {
    m_.right[slot][eq] = (float)((double)m_.right[slot][eq] + val);
    m_.net[slot][eq] = (float)((double)m_.net[slot][eq] + val);
  }
}

void Parser::term_list(int side) {
  bool first = true;
  for (;;) {
    std::string sign = "+";
    if (at(T_SIGN)) sign = take().text;
    else if (!first) break;
    std::string coef = "1";
    if (at(T_COEF)) coef = take().text;
    if (!at(T_ID)) { sc_.error("missing species after '" + coef + "'"); return; }
    process_term(side, sign, coef, take().text);
    first = false;
  }
}

void Parser::store_rate(const std::string& rate, const std::string& tag) {
  Reaction r;
  r.rate = rate;
  r.tag = tag;
  if (photo_) {
    r.kind = RATE_PHOTO;
    photo_ = false;
  } else {
    // A bare number (nothing but blanks after it) is a constant rate.
    const char* s = rate.c_str();
    char* end = nullptr;
    double v = std::strtod(s, &end);
    bool number = end != s;
    if (number)
      for (const char* q = end; *q; q++)
        if (!std::isspace((unsigned char)*q)) number = false;
    if (number) {
      r.kind = RATE_NUMBER;
      r.number = (float)v;
    } else {
      r.kind = RATE_EXPRESSION;
    }
  }
  m_.reactions.push_back(r);
}

void Parser::equation() {
  std::string tag;
  if (at(T_LT)) {
    take();
    if (at(T_TAG)) tag = take().text;
    if (at(T_GT)) take();
    else sc_.error("missing '>' after equation tag");
  }
  photo_ = false;
  term_list(0);
  if (!at(T_EQ)) { recover(); return; }
  take();
  term_list(1);
  if (!at(T_COLON)) { recover(); return; }
  take();
  std::string rate;
  while (at(T_RATE)) rate += take().text;
  if (rate.empty()) sc_.error("missing rate");
  // the stoichiometry vectors of every slot cover this equation
  int eq = (int)m_.reactions.size();
  for (size_t s = 0; s < m_.order.size(); s++)
    for (auto* v : {&m_.left[s], &m_.right[s], &m_.net[s]})
      if ((int)v->size() <= eq) v->resize(eq + 1, 0.0f);
  store_rate(rate, tag);
}

void Parser::equation_list() {
  while (at(T_LT) || at(T_SIGN) || at(T_COEF) || at(T_ID)) {
    equation();
    if (at(T_SEMI)) skip_semicolons();
    else if (!at(T_END) && !at(T_CMD)) recover();
  }
}

void Parser::inline_block() {
  if (!at(T_INLCTX)) { sc_.error("#INLINE needs a context"); return; }
  std::string ctx = take().text;
  std::string code;
  while (at(T_INLTEXT)) code += take().text;
  if (!at(T_INLEND)) { sc_.error("missing #ENDINLINE"); return; }
  take();
  std::string key;
  for (char ch : ctx) key += (char)std::toupper((unsigned char)ch);
  m_.inline_code[key] += code;
}

}  // namespace

bool parse_mechanism(const std::string& path, const std::string& kpp_home, Mechanism& m) {
  std::string dir = ".";
  size_t slash = path.rfind('/');
  if (slash != std::string::npos) dir = path.substr(0, slash);
  Scanner sc(m, kpp_home, dir);
  if (!sc.open(path)) {
    std::fprintf(stderr, "kppcu: cannot read %s\n", path.c_str());
    return false;
  }
  Parser p(m, sc);
  p.run();
  // every stoichiometry vector spans all reactions
  int nr = m.nreact();
  for (size_t s = 0; s < m.order.size(); s++)
    for (auto* v : {&m.left[s], &m.right[s], &m.net[s]}) v->resize(nr, 0.0f);
  return m.errors == 0;
}

}  // namespace kppcu
