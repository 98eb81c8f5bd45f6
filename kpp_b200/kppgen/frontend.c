/* Hand-written scanner and parser for the KPP mechanism language.
 *
 * KPP's generator (the C sources in src/) is written against a flex scanner
 * (src/scan.l) and a bison parser (src/scan.y).  flex, bison and libfl are not
 * installed in this image, so the generator cannot be built from its own
 * Makefile (src/Makefile:38-54,86-93).  This file supplies the symbols that
 * lex.yy.c and y.tab.c would provide, so that the unchanged sources in src/
 * (scanner.c, kpp.c, gen.c, code*.c, ...) link into a working `kpp` binary.
 * Two builds use it: the oracle's reference generator (oracle/build_ref.sh,
 * the reference's own generated C code, for tests and the CPU baseline) and
 * the generator with kpp_b200's CUDA target (kpp_b200/kppgen/build.py).
 *
 * Behaviour followed:
 *   - start conditions, patterns and actions of src/scan.l:37-298: flex
 *     semantics (longest match, earliest rule on a tie, %s states inclusive of
 *     the unprefixed rules, INL_CODE exclusive), the single `oldstate` slot for
 *     comments, and the include stack of src/scan.l:344-390;
 *   - the keyword table of src/scan.l:301-341;
 *   - the grammar and semantic actions of src/scan.y:105-372, parsed here by
 *     recursive descent with one token of lookahead, with the semantic
 *     actions called at the same points as the LALR reductions (an action
 *     runs before the token that follows its construct is scanned past);
 *   - error messages of src/scan.y:374-442 (ParserErrorMessage) and the
 *     Parser() entry of src/scan.y:445-466.
 */
#include <ctype.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gdata.h"
#include "scan.h"
#include "y.tab.h"

/* ---- globals that lex.yy.c / y.tab.c define in the reference build ---- */
int crt_line_no = 1;
char *crt_filename;
char crtToken[MAX_K];
char nextToken[MAX_K];
int crtTokType;
int nextTokType;
int crtLine;
char crtFile[MAX_K];
int nError = 0;
int nWarning = 0;
int crt_section;
int eqState;
int isPhoto = 0;
int yyerrflag = 0;

/* ---------------------------------------------------------------------- */
/* Scanner                                                                 */
/* ---------------------------------------------------------------------- */

enum lex_state {
  S_INITIAL, S_CMD, S_INC, S_MOD, S_INT, S_PRM, S_DSP, S_SSP, S_INI, S_EQN,
  S_EQNTAG, S_RATE, S_FAM, S_CR_IGNORE, S_SC_IGNORE, S_ATM, S_LKT, S_INL,
  S_MNI, S_TPT, S_USE, S_COMMENT, S_COMMENT2, S_EQN_ID, S_INL_CODE
};

#define MAX_INCLUDE 10

typedef struct {
  char *text;     /* whole file contents */
  size_t len;
  size_t pos;
  int line;       /* saved crt_line_no of the including file */
  char *name;     /* saved crt_filename of the including file */
} source_t;

static source_t src_stack[MAX_INCLUDE + 1];
static int src_depth = -1;      /* index of the active source */
static int lex_state_cur = S_INITIAL;
static int lex_oldstate = S_INITIAL;

typedef struct {
  const char *name;
  int next;
  int cmd;
} keyword_t;

/* src/scan.l:301-341 */
static const keyword_t keyword_table[] = {
  {"INCLUDE", S_INC, 0},          {"MODEL", S_MOD, 0},
  {"INTEGRATOR", S_INT, 0},       {"JACOBIAN", S_PRM, JACOBIAN},
  {"HESSIAN", S_PRM, HESSIAN},    {"DECLARE", S_PRM, DECLARE},
  {"STOICMAT", S_PRM, STOICMAT},  {"STOCHASTIC", S_PRM, STOCHASTIC},
  {"DOUBLE", S_PRM, DOUBLE},      {"REORDER", S_PRM, REORDER},
  {"MEX", S_PRM, MEX},            {"DUMMYINDEX", S_PRM, DUMMYINDEX},
  {"EQNTAGS", S_PRM, EQNTAGS},    {"FUNCTION", S_PRM, FUNCTION},
  {"ATOMS", S_ATM, ATOMDECL},     {"CHECK", S_ATM, CHECK},
  {"CHECKALL", S_INITIAL, CHECKALL}, {"DEFVAR", S_DSP, DEFVAR},
  {"DEFFIX", S_DSP, DEFFIX},      {"SETVAR", S_SSP, SETVAR},
  {"SETFIX", S_SSP, SETFIX},      {"INITVALUES", S_INI, INITVALUES},
  {"EQUATIONS", S_EQN, EQUATIONS}, {"FAMILIES", S_FAM, FAMILIES},
  {"LOOKAT", S_LKT, LOOKAT},      {"LOOKATALL", S_INITIAL, LOOKATALL},
  {"MONITOR", S_MNI, MONITOR},    {"WRITE_ATM", S_INITIAL, WRITE_ATM},
  {"WRITE_SPC", S_INITIAL, WRITE_SPC}, {"WRITE_MAT", S_INITIAL, WRITE_MAT},
  {"LANGUAGE", S_PRM, LANGUAGE},  {"INLINE", S_INL, INLINE},
  {"ENDINLINE", S_INITIAL, ENDINLINE}, {"INTFILE", S_PRM, INTFILE},
  {"DRIVER", S_PRM, DRIVER},      {"FLUX", S_PRM, FLUX},
  {"UPPERCASEF90", S_PRM, UPPERCASEF90}, {"MINVERSION", S_PRM, MINVERSION},
  {"AUTOREDUCE", S_PRM, AUTOREDUCE}, {"GRAPH", S_PRM, GRAPH},
  {NULL, 0, 0}};

int EqNoCase(char *s1, char *s2) {
  while (*s1) {
    if (toupper((unsigned char)*s1++) != toupper((unsigned char)*s2++)) return 0;
  }
  return *s1 == *s2;
}

static int check_keyword(char *cmd) {
  int i;
  for (i = 0; keyword_table[i].name; i++)
    if (EqNoCase(cmd, (char *)keyword_table[i].name)) return i;
  ScanError("'%s': Unknown command (ignored)", cmd);
  return -1;
}

static char *read_whole_file(const char *name, size_t *len) {
  FILE *f = fopen(name, "rb");
  char *buf;
  long n;
  if (!f) return NULL;
  fseek(f, 0, SEEK_END);
  n = ftell(f);
  fseek(f, 0, SEEK_SET);
  buf = (char *)malloc((size_t)n + 1);
  if (n > 0 && fread(buf, 1, (size_t)n, f) != (size_t)n) {
    fclose(f);
    free(buf);
    return NULL;
  }
  buf[n] = 0;
  fclose(f);
  *len = (size_t)n;
  return buf;
}

/* src/scan.l:344-371 */
static void include_file(char *name) {
  size_t len = 0;
  char *text;
  if (src_depth + 1 > MAX_INCLUDE) {
    printf("\nInclude nested too deep. Include %s ignored", name);
    return;
  }
  text = read_whole_file(name, &len);
  if (!text) FatalError(3, "%s: Can't read file", name);
  src_depth++;
  src_stack[src_depth].text = text;
  src_stack[src_depth].len = len;
  src_stack[src_depth].pos = 0;
  src_stack[src_depth].line = crt_line_no;
  src_stack[src_depth].name = crt_filename;
  crt_line_no = 1;
  crt_filename = (char *)malloc(strlen(name) + 1);
  strcpy(crt_filename, name);
}

/* src/scan.l:373-390; returns 1 when an included file was closed */
static int end_include(void) {
  if (src_depth > 0) {
    free(src_stack[src_depth].text);
    free(crt_filename);
    crt_line_no = src_stack[src_depth].line;
    crt_filename = src_stack[src_depth].name;
    src_depth--;
    return 1;
  }
  return 0;
}

/* ---- pattern matchers: length of the longest match at p, 0 = none ---- */
static size_t m_space(const char *p, size_t n) {
  size_t i = 0;
  while (i < n && (p[i] == ' ' || p[i] == '\t')) i++;
  return i;
}
static size_t m_ch(const char *p, size_t n, char c) { return (n > 0 && p[0] == c) ? 1 : 0; }
static size_t m_until(const char *p, size_t n, const char *stop) {
  size_t i = 0;
  while (i < n && !strchr(stop, p[i])) i++;
  return i;
}
/* STRING [^ \t\n{}#;]+ */
static size_t m_string(const char *p, size_t n) { return m_until(p, n, " \t\n{}#;"); }
static int is_lit(char c) { return isalpha((unsigned char)c) || c == '_'; }
static int is_alnum_(char c) { return isalnum((unsigned char)c) || c == '_'; }
/* IDSPC {LIT}[a-zA-Z_0-9]* */
static size_t m_idspc(const char *p, size_t n) {
  size_t i;
  if (n == 0 || !is_lit(p[0])) return 0;
  for (i = 1; i < n && is_alnum_(p[i]); i++) {}
  return i;
}
/* TAG [a-zA-Z_0-9]+ */
static size_t m_tag(const char *p, size_t n) {
  size_t i = 0;
  while (i < n && is_alnum_(p[i])) i++;
  return i;
}
/* NR {CIF}* */
static size_t m_nr(const char *p, size_t n) {
  size_t i = 0;
  while (i < n && isdigit((unsigned char)p[i])) i++;
  return i;
}
/* NRS [+-]?{CIF}+ */
static size_t m_nrs(const char *p, size_t n) {
  size_t i = 0, d;
  if (i < n && (p[i] == '+' || p[i] == '-')) i++;
  d = m_nr(p + i, n - i);
  return d ? i + d : 0;
}
/* STOICH {LIT}[a-zA-Z_0-9]*[*] */
static size_t m_stoich(const char *p, size_t n) {
  size_t i = m_idspc(p, n);
  return (i && i < n && p[i] == '*') ? i + 1 : 0;
}
static size_t m_exponent(const char *p, size_t n) {
  size_t e;
  if (n == 0 || !strchr("eEdD", p[0])) return 0;
  e = m_nrs(p + 1, n - 1);
  return e ? 1 + e : 0;
}
/* FLOAT {REAL}([eEdD]{NRS})?  with REAL {NRS}?"."?{NR} */
static size_t m_float(const char *p, size_t n) {
  size_t i = m_nrs(p, n);
  if (i < n && p[i] == '.') i++;
  i += m_nr(p + i, n - i);
  return i + m_exponent(p + i, n - i);
}
/* UFLOAT {UREAL}([eEdD]{NRS})?  with UREAL {NR}?"."?{NR} */
static size_t m_ufloat(const char *p, size_t n) {
  size_t i = m_nr(p, n);
  if (i < n && p[i] == '.') i++;
  i += m_nr(p + i, n - i);
  return i + m_exponent(p + i, n - i);
}

/* Rules in the order of src/scan.l.  `st` is the start condition a rule is
 * prefixed with, or -1 for the unprefixed rules (active in INITIAL and every
 * inclusive state, not in the exclusive INL_CODE). */
enum rule_id {
  R_SPACE, R_HASH, R_LBRACE, R_SLASH2, R_COM_BODY, R_COM_END, R_COM2_BODY,
  R_COM2_END, R_CR, R_CMD, R_INC, R_MOD, R_INT, R_PRM, R_CRIGN, R_ATM_ID,
  R_ATM_SEMI, R_EQN_STOICH, R_FAM_COLON, R_FAM_ID, R_FAM_NR, R_FAM_EQ,
  R_FAM_PLUS, R_FAM_SEMI, R_FAM_BAD, R_DSP_ID, R_DSP_NR, R_DSP_EQ, R_DSP_PLUS,
  R_DSP_SEMI, R_DSP_BAD, R_SSP_ID, R_SSP_SEMI, R_INI_ID, R_INI_EQ, R_INI_SEMI,
  R_INI_FLOAT, R_INI_BAD, R_EQN_ID, R_EQN_EQ, R_EQN_UFLOAT, R_EQN_COLON,
  R_EQN_SIGN, R_EQN_LESS, R_TAG, R_TAG_GT, R_RATE, R_RATE_SEMI, R_LKT_ID,
  R_LKT_SEMI, R_TPT_ID, R_TPT_SEMI, R_USE_STR, R_USE_SEMI, R_MNI_ID,
  R_MNI_SEMI, R_INL_CTX, R_INLC_HASH, R_INLC_NL, R_INLC_BODY, R_COUNT
};

static const int rule_state[R_COUNT] = {
  -1, -1, -1, -1, S_COMMENT, S_COMMENT, S_COMMENT2, S_COMMENT2, -1, S_CMD,
  S_INC, S_MOD, S_INT, S_PRM, S_CR_IGNORE, S_ATM, S_ATM, S_EQN, S_FAM, S_FAM,
  S_FAM, S_FAM, S_FAM, S_FAM, S_FAM, S_DSP, S_DSP, S_DSP, S_DSP, S_DSP, S_DSP,
  S_SSP, S_SSP, S_INI, S_INI, S_INI, S_INI, S_INI, S_EQN, S_EQN, S_EQN, S_EQN,
  S_EQN, S_EQN, S_EQNTAG, S_EQNTAG, S_RATE, S_RATE, S_LKT, S_LKT, S_TPT,
  S_TPT, S_USE, S_USE, S_MNI, S_MNI, S_INL, S_INL_CODE, S_INL_CODE, S_INL_CODE};

static size_t rule_match(int r, const char *p, size_t n) {
  switch (r) {
    case R_SPACE: return m_space(p, n);
    case R_HASH: return m_ch(p, n, '#');
    case R_LBRACE: return m_ch(p, n, '{');
    case R_SLASH2: return (n >= 2 && p[0] == '/' && p[1] == '/') ? 2 : 0;
    case R_COM_BODY: return m_until(p, n, "}\n");
    case R_COM_END: return m_ch(p, n, '}');
    case R_COM2_BODY: return m_until(p, n, "\n");
    case R_COM2_END: return m_ch(p, n, '\n');
    case R_CR: return m_ch(p, n, '\n');
    case R_CMD: case R_INC: case R_MOD: case R_INT: case R_PRM: case R_CRIGN:
    case R_RATE: case R_USE_STR: case R_INL_CTX:
      return m_string(p, n);
    case R_ATM_ID: case R_FAM_ID: case R_DSP_ID: case R_SSP_ID: case R_INI_ID:
    case R_EQN_ID: case R_LKT_ID: case R_TPT_ID: case R_MNI_ID:
      return m_idspc(p, n);
    case R_ATM_SEMI: case R_FAM_SEMI: case R_DSP_SEMI: case R_SSP_SEMI:
    case R_INI_SEMI: case R_RATE_SEMI: case R_LKT_SEMI: case R_TPT_SEMI:
    case R_USE_SEMI: case R_MNI_SEMI:
      return m_ch(p, n, ';');
    case R_EQN_STOICH: return m_stoich(p, n);
    case R_FAM_COLON: case R_EQN_COLON: return m_ch(p, n, ':');
    case R_FAM_NR: case R_DSP_NR: return m_nr(p, n);
    case R_FAM_EQ: case R_DSP_EQ: case R_INI_EQ: case R_EQN_EQ: return m_ch(p, n, '=');
    case R_FAM_PLUS: case R_DSP_PLUS: return m_ch(p, n, '+');
    case R_FAM_BAD: case R_DSP_BAD: return (n > 0 && p[0] != ';' && p[0] != '#') ? 1 : 0;
    case R_INI_FLOAT: return m_float(p, n);
    case R_INI_BAD: return (n > 0 && !strchr("=;#", p[0])) ? 1 : 0;
    case R_EQN_UFLOAT: return m_ufloat(p, n);
    case R_EQN_SIGN: return (n > 0 && (p[0] == '+' || p[0] == '-')) ? 1 : 0;
    case R_EQN_LESS: return m_ch(p, n, '<');
    case R_TAG: return m_tag(p, n);
    case R_TAG_GT: return m_ch(p, n, '>');
    case R_INLC_HASH: {
      size_t i;
      if (n == 0 || p[0] != '#') return 0;
      for (i = 1; i < n && p[i] != ' ' && p[i] != '\t' && p[i] != '\n'; i++) {}
      return i;
    }
    case R_INLC_NL: return m_ch(p, n, '\n');
    case R_INLC_BODY: return m_until(p, n, "#\n");
  }
  return 0;
}

static int rule_active(int r, int st) {
  if (rule_state[r] == -1) return st != S_INL_CODE;
  return rule_state[r] == st;
}

typedef struct {
  int type;
  char text[MAX_K];
} token_t;

static char yytext_buf[MAX_K];

/* Bookkeeping of the RETURN macro, src/scan.l:85-97 */
static int lex_return(token_t *t, int type) {
  if (yyerrflag == 0) {
    strcpy(crtToken, nextToken);
    crtTokType = nextTokType;
    crtLine = crt_line_no;
    strcpy(crtFile, crt_filename);
  }
  strcpy(nextToken, yytext_buf);
  nextTokType = type;
  t->type = type;
  return type;
}

static void copy_text(char *dst, const char *p, size_t len) {
  if (len >= MAX_K) len = MAX_K - 1;
  memcpy(dst, p, len);
  dst[len] = 0;
}

static int lex_next(token_t *t) {
  for (;;) {
    source_t *s = &src_stack[src_depth];
    const char *p = s->text + s->pos;
    size_t n = s->len - s->pos;
    size_t best_len = 0;
    int best = -1, r;

    if (n == 0) {
      if (!end_include()) {
        yytext_buf[0] = 0;
        t->text[0] = 0;
        return lex_return(t, TK_EOF);
      }
      continue;
    }
    for (r = 0; r < R_COUNT; r++) {
      size_t len;
      if (!rule_active(r, lex_state_cur)) continue;
      len = rule_match(r, p, n);
      if (len > best_len) {
        best_len = len;
        best = r;
      }
    }
    if (best < 0) {
      /* flex default rule: echo the unmatched character */
      putchar(p[0]);
      s->pos++;
      continue;
    }
    copy_text(yytext_buf, p, best_len);
    s->pos += best_len;
    strcpy(t->text, yytext_buf);

    switch (best) {
      case R_SPACE: break;
      case R_HASH: lex_state_cur = S_CMD; break;
      case R_LBRACE: lex_oldstate = lex_state_cur; lex_state_cur = S_COMMENT; break;
      case R_SLASH2: lex_oldstate = lex_state_cur; lex_state_cur = S_COMMENT2; break;
      case R_COM_BODY: break;
      case R_COM_END: lex_state_cur = lex_oldstate; break;
      case R_COM2_BODY: break;
      case R_COM2_END: crt_line_no++; lex_state_cur = lex_oldstate; break;
      case R_CR: crt_line_no++; break;
      case R_CMD: {
        int idx = check_keyword(yytext_buf);
        if (idx < 0) {
          lex_state_cur = S_CR_IGNORE;
          break;
        }
        lex_state_cur = keyword_table[idx].next;
        if (keyword_table[idx].cmd) {
          crt_section = keyword_table[idx].cmd;
          return lex_return(t, keyword_table[idx].cmd);
        }
        break;
      }
      case R_INC: include_file(IncName(yytext_buf)); lex_state_cur = S_CR_IGNORE; break;
      case R_MOD: include_file(ModelName(yytext_buf)); lex_state_cur = S_CR_IGNORE; break;
      case R_INT: include_file(IntegName(yytext_buf)); lex_state_cur = S_CR_IGNORE; break;
      case R_PRM: lex_state_cur = S_CR_IGNORE; return lex_return(t, PARAMETER);
      case R_CRIGN: ScanError("Extra parameter on command line '%s'", yytext_buf); break;
      case R_ATM_ID: return lex_return(t, ATOMID);
      case R_EQN_STOICH: return lex_return(t, EQNCOEF);
      case R_FAM_COLON: return lex_return(t, FAMCOLON);
      case R_FAM_ID: case R_DSP_ID: return lex_return(t, SPCSPC);
      case R_FAM_NR: case R_DSP_NR: return lex_return(t, SPCNR);
      case R_FAM_EQ: case R_DSP_EQ: return lex_return(t, SPCEQUAL);
      case R_FAM_PLUS: case R_DSP_PLUS: return lex_return(t, SPCPLUS);
      case R_ATM_SEMI: case R_FAM_SEMI: case R_DSP_SEMI: case R_SSP_SEMI:
      case R_INI_SEMI: case R_LKT_SEMI: case R_TPT_SEMI: case R_USE_SEMI:
      case R_MNI_SEMI:
        return lex_return(t, ';');
      case R_FAM_BAD: case R_DSP_BAD:
        ScanError("Invalid character '%c' in species definition", yytext_buf[0]);
        break;
      case R_SSP_ID: return lex_return(t, SSPID);
      case R_INI_ID: return lex_return(t, INISPC);
      case R_INI_EQ: return lex_return(t, INIEQUAL);
      case R_INI_FLOAT: return lex_return(t, INIVALUE);
      case R_INI_BAD:
        ScanError("Invalid character '%c' in initial values", yytext_buf[0]);
        break;
      case R_EQN_ID: return lex_return(t, EQNSPC);
      case R_EQN_EQ: return lex_return(t, EQNEQUAL);
      case R_EQN_UFLOAT: return lex_return(t, EQNCOEF);
      case R_EQN_COLON: lex_state_cur = S_RATE; return lex_return(t, EQNCOLON);
      case R_EQN_SIGN: return lex_return(t, EQNSIGN);
      case R_EQN_LESS: lex_state_cur = S_EQNTAG; return lex_return(t, EQNLESS);
      case R_TAG: return lex_return(t, EQNTAG);
      case R_TAG_GT: lex_state_cur = S_EQN; return lex_return(t, EQNGREATER);
      case R_RATE: return lex_return(t, RATE);
      case R_RATE_SEMI: lex_state_cur = S_EQN; return lex_return(t, ';');
      case R_LKT_ID: return lex_return(t, LKTID);
      case R_TPT_ID: return lex_return(t, TPTID);
      case R_USE_STR: return lex_return(t, USEID);
      case R_MNI_ID: return lex_return(t, MNIID);
      case R_INL_CTX: lex_state_cur = S_INL_CODE; return lex_return(t, INLCTX);
      case R_INLC_HASH:
        if (EqNoCase(yytext_buf + 1, "ENDINLINE")) {
          lex_state_cur = S_INITIAL;
          return lex_return(t, ENDINLINE);
        }
        return lex_return(t, INCODE);
      case R_INLC_NL: crt_line_no++; return lex_return(t, INCODE);
      case R_INLC_BODY: return lex_return(t, INCODE);
    }
  }
}

int yylex(void) {
  token_t t;
  return lex_next(&t);
}

/* ---------------------------------------------------------------------- */
/* Parser                                                                  */
/* ---------------------------------------------------------------------- */

static token_t look;       /* one token of lookahead */
static int have_look = 0;

static token_t *peek(void) {
  if (!have_look) {
    lex_next(&look);
    have_look = 1;
  }
  return &look;
}

static token_t take(void) {
  token_t t = *peek();
  have_look = 0;
  return t;
}

/* src/scan.y:374-442 */
static void parser_error_message(void) {
  if (crtToken[0] == ';') {
    ParserError("Misplaced ';'");
    return;
  }
  switch (crtTokType) {
    case ATOMID: ParserError("Missing ';' after '%s'", crtToken); break;
    case SPCSPC: ParserError("Missing ';' or '+' after '%s'", crtToken); break;
    case SPCNR: ParserError("Missing species after '%s'", crtToken); break;
    case SPCPLUS: ParserError("Missing atom after '%s'", crtToken); break;
    case SPCEQUAL: ParserError("Invalid '=' after '%s'", crtToken); break;
    case INISPC: ParserError("Missing '=' after '%s'", crtToken); break;
    case INIEQUAL: ParserError("Missing value after '%s'", crtToken); break;
    case INIVALUE: ParserError("Missing ';' after '%s'", crtToken); break;
    case EQNSPC: ParserError("Missing '+' or '=' after '%s'", crtToken); break;
    case EQNEQUAL: ParserError("Invalid right hand side of equation"); break;
    case EQNCOLON: ParserError("Missing rate after '%s'", crtToken); break;
    case EQNSIGN: ParserError("Missing coeficient after '%s'", crtToken); break;
    case EQNCOEF: ParserError("Missing species after '%s'", crtToken); break;
    case RATE: ParserError("Missing ';' after '%s'", crtToken); break;
    case INLINE: ParserError("Missing inline option after '%s'", crtToken); break;
    default: ParserError("Syntax error after '%s'", crtToken);
  }
}

static int is_section_start(int type) {
  switch (type) {
    case JACOBIAN: case HESSIAN: case DECLARE: case STOICMAT: case DOUBLE:
    case REORDER: case MEX: case DUMMYINDEX: case EQNTAGS: case FUNCTION:
    case STOCHASTIC: case ATOMDECL: case CHECK: case DEFVAR: case DEFFIX:
    case SETVAR: case SETFIX: case INITVALUES: case EQUATIONS: case FAMILIES:
    case LOOKAT: case MONITOR: case CHECKALL: case LOOKATALL: case WRITE_ATM:
    case WRITE_SPC: case WRITE_MAT: case LANGUAGE: case INLINE: case INTFILE:
    case DRIVER: case FLUX: case AUTOREDUCE: case UPPERCASEF90: case MINVERSION:
    case GRAPH: case TK_EOF:
      return 1;
  }
  return 0;
}

/* Error recovery of the `error semicolon` productions: report, then drop
 * tokens up to and including the next ';' (or stop at a new section). */
static void recover_to_semicolon(void) {
  parser_error_message();
  while (!is_section_start(peek()->type) && peek()->type != ';') take();
  if (peek()->type == ';') take();
  while (peek()->type == ';') take();
}

/* semicolon : semicolon ';' | ';'   (src/scan.y:203-207) */
static int semicolon(void) {
  if (peek()->type != ';') return 0;
  take();
  while (peek()->type == ';') {
    ScanWarning("Unnecessary ';'");
    take();
  }
  return 1;
}

static int expect(int type, token_t *out) {
  if (peek()->type != type) return 0;
  *out = take();
  return 1;
}

/* A list section: items while the lookahead can start one. */
typedef int (*item_fn)(void);

static void parse_list(item_fn item, int first_type) {
  int count = 0;
  for (;;) {
    int t = peek()->type;
    if (count > 0 && is_section_start(t)) return;
    if (t == TK_EOF) {
      if (count == 0) parser_error_message();
      return;
    }
    if (t != first_type || !item() || !semicolon()) {
      recover_to_semicolon();
    }
    count++;
  }
}

/* atomdef (src/scan.y:213-219) */
static int item_atom(void) {
  token_t id = take();
  switch (crt_section) {
    case ATOMDECL: DeclareAtom(id.text); break;
    case CHECK: SetAtomType(id.text, DO_CHECK); break;
  }
  return 1;
}

static int item_lookat(void) {
  token_t id = take();
  AddLookAt(id.text);
  return 1;
}

static int item_monitor(void) {
  token_t id = take();
  AddMonitor(id.text);
  return 1;
}

/* setspcspc (src/scan.y:239-245) */
static int item_setspc(void) {
  token_t id = take();
  switch (crt_section) {
    case SETVAR: SetSpcType(VAR_SPC, id.text); break;
    case SETFIX: SetSpcType(FIX_SPC, id.text); break;
  }
  return 1;
}

/* atom : SPCNR SPCSPC | SPCSPC   (src/scan.y:300-306), used for atoms and
 * family members */
static int atom_or_member(int member) {
  token_t nr, name;
  if (peek()->type == SPCNR) {
    nr = take();
    if (!expect(SPCSPC, &name)) return 0;
    if (member) AddMember(name.text, nr.text);
    else AddAtom(name.text, nr.text);
    return 1;
  }
  if (!expect(SPCSPC, &name)) return 0;
  if (member) AddMember(name.text, "1");
  else AddAtom(name.text, "1");
  return 1;
}

/* spc : spcname | spcdef   (src/scan.y:277-296) */
static int item_species(void) {
  token_t name = take();
  if (peek()->type == SPCEQUAL) {
    take();
    if (!atom_or_member(0)) return 0;
    while (peek()->type == SPCPLUS) {
      take();
      if (!atom_or_member(0)) return 0;
    }
  }
  switch (crt_section) {
    case DEFVAR: DeclareSpecies(VAR_SPC, name.text); break;
    case DEFFIX: DeclareSpecies(FIX_SPC, name.text); break;
  }
  return 1;
}

/* family : SPCSPC FAMCOLON members   (src/scan.y:252-265) */
static int item_family(void) {
  token_t name = take();
  token_t colon;
  if (!expect(FAMCOLON, &colon)) return 0;
  if (!atom_or_member(1)) return 0;
  while (peek()->type == SPCPLUS) {
    take();
    if (!atom_or_member(1)) return 0;
  }
  DeclareFamily(name.text);
  return 1;
}

/* assignment : INISPC INIEQUAL INIVALUE   (src/scan.y:313-315) */
static int item_initvalue(void) {
  token_t spc = take(), eq, val;
  if (!expect(INIEQUAL, &eq)) return 0;
  if (!expect(INIVALUE, &val)) return 0;
  AssignInitialValue(spc.text, val.text);
  return 1;
}

static char crt_term[30];
static char crt_coef[30];

/* term : EQNCOEF EQNSPC | EQNSPC   (src/scan.y:363-371) */
static int term(void) {
  token_t coef, spc;
  if (peek()->type == EQNCOEF) {
    coef = take();
    if (!expect(EQNSPC, &spc)) return 0;
    strncpy(crt_term, spc.text, sizeof crt_term - 1);
    strncpy(crt_coef, coef.text, sizeof crt_coef - 1);
    return 1;
  }
  if (!expect(EQNSPC, &spc)) return 0;
  strncpy(crt_term, spc.text, sizeof crt_term - 1);
  strcpy(crt_coef, "1");
  return 1;
}

/* expresion (src/scan.y:352-362) */
static int expression(void) {
  token_t sign;
  if (peek()->type == EQNSIGN) {
    sign = take();
    if (!term()) return 0;
    ProcessTerm(eqState, sign.text, crt_coef, crt_term);
  } else {
    if (!term()) return 0;
    ProcessTerm(eqState, "+", crt_coef, crt_term);
  }
  while (peek()->type == EQNSIGN) {
    sign = take();
    if (!term()) return 0;
    ProcessTerm(eqState, sign.text, crt_coef, crt_term);
  }
  return 1;
}

/* equation (src/scan.y:316-351) */
static int item_equation(void) {
  char tag[MAX_K];
  char rate[MAX_K];
  token_t t;
  int tagged = 0;
  if (peek()->type == EQNLESS) {
    take();
    if (!expect(EQNTAG, &t)) return 0;
    strcpy(tag, t.text);
    if (!expect(EQNGREATER, &t)) return 0;
    tagged = 1;
  }
  if (!expression()) return 0;
  if (!expect(EQNEQUAL, &t)) return 0;
  eqState = RHS;
  if (!expression()) return 0;
  if (!expect(EQNCOLON, &t)) return 0;
  ProcessTerm(eqState, "+", "1", "RR");
  eqState = RAT;
  if (peek()->type != RATE) return 0;
  rate[0] = 0;
  while (peek()->type == RATE) {
    t = take();
    if (strlen(rate) + strlen(t.text) < MAX_K) strcat(rate, t.text);
  }
  eqState = LHS;
  StoreEquationRate(rate, tagged ? tag : "          ");
  CheckEquation();
  return 1;
}

static int equation_start(int t) {
  return t == EQNLESS || t == EQNSIGN || t == EQNCOEF || t == EQNSPC;
}

static void parse_equations(void) {
  int count = 0;
  for (;;) {
    int t = peek()->type;
    if (count > 0 && is_section_start(t)) return;
    if (t == TK_EOF) return;
    if (!equation_start(t) || !item_equation() || !semicolon()) {
      recover_to_semicolon();
      eqState = LHS;
    }
    count++;
  }
}

static void parse_parameter_cmd(void (*cmd)(char *)) {
  token_t prm;
  if (!expect(PARAMETER, &prm)) {
    parser_error_message();
    return;
  }
  cmd(prm.text);
}

/* INLINE INLCTX inlinecode ENDINLINE   (src/scan.y:179-186) */
static void parse_inline(void) {
  token_t ctx, t;
  char *buf = NULL;
  int buflen = 0;
  if (!expect(INLCTX, &ctx)) {
    parser_error_message();
    return;
  }
  while (peek()->type == INCODE) {
    t = take();
    if (!buf) {
      buf = (char *)malloc(MAX_INLINE);
      buflen = MAX_INLINE;
      strcpy(buf, t.text);
    } else {
      buf = AppendString(buf, t.text, &buflen, MAX_INLINE);
    }
  }
  if (!expect(ENDINLINE, &t) || !buf) {
    parser_error_message();
    free(buf);
    return;
  }
  AddInlineCode(ctx.text, buf);
  free(buf);
}

/* section (src/scan.y:108-202) */
static void parse_section(void) {
  token_t t = take();
  switch (t.type) {
    case JACOBIAN: parse_parameter_cmd(CmdJacobian); break;
    case HESSIAN: parse_parameter_cmd(CmdHessian); break;
    case DECLARE: parse_parameter_cmd(CmdDeclareValues); break;
    case STOICMAT: parse_parameter_cmd(CmdStoicmat); break;
    case DOUBLE: parse_parameter_cmd(CmdDouble); break;
    case REORDER: parse_parameter_cmd(CmdReorder); break;
    case MEX: parse_parameter_cmd(CmdMex); break;
    case DUMMYINDEX: parse_parameter_cmd(CmdDummyindex); break;
    case EQNTAGS: parse_parameter_cmd(CmdEqntags); break;
    case FUNCTION: parse_parameter_cmd(CmdFunction); break;
    case STOCHASTIC: parse_parameter_cmd(CmdStochastic); break;
    case LANGUAGE: parse_parameter_cmd(CmdLanguage); break;
    case INTFILE: parse_parameter_cmd(CmdIntegrator); break;
    case DRIVER: parse_parameter_cmd(CmdDriver); break;
    case FLUX: parse_parameter_cmd(CmdFlux); break;
    case AUTOREDUCE: parse_parameter_cmd(CmdAutoReduce); break;
    case UPPERCASEF90: parse_parameter_cmd(CmdUpperCaseF90); break;
    case MINVERSION: parse_parameter_cmd(CmdMinVersion); break;
    case GRAPH: parse_parameter_cmd(CmdGraph); break;
    case ATOMDECL: case CHECK: parse_list(item_atom, ATOMID); break;
    case DEFVAR: case DEFFIX: parse_list(item_species, SPCSPC); break;
    case SETVAR: case SETFIX: parse_list(item_setspc, SSPID); break;
    case INITVALUES: parse_list(item_initvalue, INISPC); break;
    case EQUATIONS: parse_equations(); break;
    case FAMILIES: parse_list(item_family, SPCSPC); break;
    case LOOKAT: parse_list(item_lookat, LKTID); break;
    case MONITOR: parse_list(item_monitor, MNIID); break;
    case CHECKALL: CheckAll(); break;
    case LOOKATALL: LookAtAll(); break;
    case WRITE_ATM: WriteAtoms(); break;
    case WRITE_SPC: WriteSpecies(); break;
    case WRITE_MAT: WriteMatrices(); break;
    case INLINE: parse_inline(); break;
    default: parser_error_message(); break;
  }
}

/* src/scan.y:445-466 */
int Parser(char *filename) {
  size_t len = 0;
  char *text;
  crt_filename = filename;
  text = read_whole_file(crt_filename, &len);
  if (!text) FatalError(7, "%s: File not found", crt_filename);
  src_depth = 0;
  src_stack[0].text = text;
  src_stack[0].len = len;
  src_stack[0].pos = 0;
  src_stack[0].line = 1;
  src_stack[0].name = filename;
  lex_state_cur = S_INITIAL;
  have_look = 0;
  nError = 0;
  nWarning = 0;
  while (peek()->type != TK_EOF) parse_section();
  free(src_stack[0].text);
  src_depth = -1;
  return nError;
}
