/* Token codes for the hand-written KPP front end (frontend.c).
 *
 * ORACLE INFRASTRUCTURE ONLY.  This header stands in for the bison-generated
 * y.tab.h that src/scanner.c includes (src/scanner.c:36).  flex, bison and
 * libfl are not installed here, so the reference generator is built with a
 * hand-written scanner/parser instead.  The token set is the one declared in
 * src/scan.y:78-101; the numeric values are this file's own.
 */
#ifndef KPP_ORACLE_YTAB_H
#define KPP_ORACLE_YTAB_H

enum kpp_oracle_token {
  TK_EOF = 0,
  JACOBIAN = 258, DOUBLE, FUNCTION, DEFVAR, DEFFIX, SETVAR, SETFIX,
  HESSIAN, STOICMAT, STOCHASTIC, DECLARE,
  INITVALUES, EQUATIONS, FAMILIES, INIEQUAL, EQNEQUAL, EQNCOLON,
  SPCPLUS, SPCEQUAL, FAMCOLON, ATOMDECL, CHECK, CHECKALL, REORDER,
  MEX, DUMMYINDEX, EQNTAGS,
  LOOKAT, LOOKATALL, MONITOR,
  WRITE_ATM, WRITE_SPC, WRITE_MAT,
  LANGUAGE, INTFILE, DRIVER, INLINE, ENDINLINE,
  PARAMETER, SPCSPC, INISPC, INIVALUE, EQNSPC, EQNSIGN, EQNCOEF,
  RATE, SPCNR, ATOMID, LKTID, MNIID, INLCTX, INCODE, SSPID,
  EQNLESS, EQNTAG, EQNGREATER,
  TPTID, USEID,
  FLUX, AUTOREDUCE, GRAPH, PLSPC, UPPERCASEF90, MINVERSION
};

#endif
