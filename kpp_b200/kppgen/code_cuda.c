/*
 * CUDA target of the KPP generator (#LANGUAGE CUDA).
 *
 * Part of kpp_b200: compiled into KPP's own generator together with its
 * unchanged sources (the src directory of KPP 3.5.0) by kpp_b200/kppgen/build.py, which
 * adds this writer beside the C, Fortran and MATLAB ones and the hooks that
 * select it: a CUDA_LANG value of `enum lang` (src/gdata.h:93), the CUDA
 * argument of #LANGUAGE (CmdLanguage, src/scanner.c:284-308) and its case in
 * Generate()'s `switch( useLang )` (src/gen.c:3905-3916).
 *
 * The mechanism's arithmetic is the C target's, text for text: the same
 * expression trees (src/code.c), the same C writers for elements, symbols,
 * assignments and constants (C_WriteElm, C_WriteAssign, ... of
 * src/code_c.c), so every Fun, Jac_SP, KppSolve and Update_RCONST statement
 * is the one the C target writes, with the same "%g" constants and the same
 * left-to-right sums.  After selecting this writer Generate() continues with
 * useLang = C_LANG, so that every C-specific decision of src/gen.c is taken as
 * for C.  What changes:
 *   - functions are device templates over their array arguments,
 *       template <class T0, ...> __device__ __forceinline__ void Fun(T0&& V, ...)
 *     so that a kernel passes thread-local arrays or strided views of
 *     per-cell work arrays in device memory;
 *   - Update_RCONST and Update_PHOTO take the generator's globals they read
 *     as arguments (RCONST, TIME, TEMP, CFACTOR, SUN and the concentrations
 *     C), one cell per call;
 *   - the sparse-structure tables of <root>_JacobianSP.cu (LU_ICOL, ...) are
 *     device arrays (__device__ const), read by the LU of the util template;
 *   - the device-side files are <root>_Function.cu, _Jacobian.cu,
 *     _JacobianSP.cu, _LinearAlgebra.cu and _Rates.cu; the util templates
 *     they paste in (sutil, blas, UserRateLaws, UpdateSun, util) come from the
 *     KPP home the build points the generator at, whose util/ holds device
 *     versions written for kpp_b200 (kpp_b200/kppgen/util/).
 * The other files (_Parameters.h, _Initialize.c, _Main.c, _Global.h, ...)
 * are the C target's host files.
 */
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include "gdata.h"
#include "code.h"

/* The C target's writers (src/code_c.c). */
void C_WriteElm( NODE * n );
void C_WriteSymbol( int op );
void C_WriteAssign( char *ls, char *rs );
void C_WriteComment( char *fmt, ... );
void C_DeclareConstant( int v, char *val );
void C_Declare( int v );
void C_ExternDeclare( int v );
void C_GlobalDeclare( int v );
void C_InitDeclare( int v, int n, void * values );

static void CUDA_InitDeclare( int v, int n, void * values )
{
  /* device copies of the sparse-structure tables; host tables elsewhere */
  if( currentFile == sparse_jacFile || currentFile == sparse_hessFile )
    bprintf( "__device__ const " );
  C_InitDeclare( v, n, values );
}

static void CUDA_FunctionStart( int f, int *vars )
{
char * name;
int narg, i;

  name = varTable[ f ]->name;
  narg = varTable[ f ]->maxi;

  if( narg == 0 && currentFile == rateFile ) {
    /* Update_RCONST, Update_PHOTO: the globals the rate expressions and the
       C_RCONST code read, as arguments */
    bprintf( "template <class TR, class TC>\n"
             "__device__ __forceinline__ void %s(\n", name );
    bprintf( "  TR&& RCONST,                           /* rate constants */\n"
             "  const double TIME,                     /* model time */\n"
             "  const double TEMP,                     /* temperature */\n"
             "  const double CFACTOR,                  /* conversion factor */\n"
             "  const double SUN,                      /* sunlight intensity */\n"
             "  TC&& C                                 /* concentrations of all species */\n"
             ")" );
    FlushBuf();
    return;
  }
  if( narg > 0 ) {
    bprintf( "template <" );
    for( i = 0; i < narg; i++ )
      bprintf( "%sclass T%d", i ? ", " : "", i );
    bprintf( ">\n" );
  }
  bprintf( "__device__ __forceinline__ void %s(\n", name );
  for( i = 0; i < narg; i++ ) {
    char arg[64];
    sprintf( arg, "T%d&& %s%s", i, varTable[ vars[ i ] ]->name, i < narg - 1 ? "," : "" );
    bprintf( "  %-38s", arg );
    if( varTable[ vars[ i ] ]->comment )
      bprintf( " /* %s */\n", varTable[ vars[ i ] ]->comment );
    else
      bprintf( "\n" );
  }
  bprintf( ")" );
  FlushBuf();
}

static void CUDA_FunctionPrototipe( int f, ... )
{
va_list args;
int i, narg, vars[ 20 ];

  narg = varTable[ f ]->maxi;
  va_start( args, f );
  for( i = 0; i < narg; i++ )
    vars[ i ] = va_arg( args, int );
  va_end( args );
  CUDA_FunctionStart( f, vars );
  bprintf( ";\n" );
  FlushBuf();
}

static void CUDA_FunctionBegin( int f, ... )
{
va_list args;
int i, narg, vars[ 20 ];

  narg = varTable[ f ]->maxi;
  va_start( args, f );
  for( i = 0; i < narg; i++ )
    vars[ i ] = va_arg( args, int );
  va_end( args );

  CommentFncBegin( f, vars );
  CUDA_FunctionStart( f, vars );
  bprintf( "\n{\n" );
  FlushBuf();
  LogFunctionComment( f, vars );
}

static void CUDA_FunctionEnd( int f )
{
  bprintf( "}\n\n" );
  FlushBuf();
  CommentFunctionEnd( f );
}

void Use_CUDA( char* rootFileName )
{
  WriteElm          = C_WriteElm;
  WriteSymbol       = C_WriteSymbol;
  WriteAssign       = C_WriteAssign;
  WriteComment      = C_WriteComment;
  DeclareConstant   = C_DeclareConstant;
  Declare           = C_Declare;
  ExternDeclare     = C_ExternDeclare;
  GlobalDeclare     = C_GlobalDeclare;
  InitDeclare       = CUDA_InitDeclare;

  FunctionStart     = CUDA_FunctionStart;
  FunctionPrototipe = CUDA_FunctionPrototipe;
  FunctionBegin     = CUDA_FunctionBegin;
  FunctionEnd       = CUDA_FunctionEnd;
  FunctionBeginNoArgDecl = NULL;

  /* device code */
  OpenFile( &functionFile, rootFileName, "_Function.cu",
            "The ODE Function of Chemical Model File (CUDA device code)" );
  OpenFile( &jacobianFile, rootFileName, "_Jacobian.cu",
            "The ODE Jacobian of Chemical Model File (CUDA device code)" );
  OpenFile( &linalgFile, rootFileName, "_LinearAlgebra.cu",
            "Linear Algebra Data and Routines File (CUDA device code)" );
  OpenFile( &rateFile, rootFileName, "_Rates.cu",
            "The Reaction Rates File (CUDA device code)" );
  if ( useJacSparse )
    OpenFile( &sparse_jacFile, rootFileName, "_JacobianSP.cu",
              "Sparse Jacobian Data Structures File (CUDA device data)" );
  if ( useHessian ) {
    OpenFile( &hessianFile, rootFileName, "_Hessian.cu", "Hessian File (CUDA device code)" );
    OpenFile( &sparse_hessFile, rootFileName, "_HessianSP.cu",
              "Sparse Hessian Data Structures File (CUDA device data)" );
  }
  /* host files, as the C target writes them */
  OpenFile( &param_headerFile, rootFileName, "_Parameters.h", "Parameter Header File" );
  OpenFile( &initFile, rootFileName, "_Initialize.c", "Initialization File" );
  OpenFile( &driverFile, rootFileName, "_Main.c", "Main Program File" );
  OpenFile( &integratorFile, rootFileName, "_Integrator.c",
            "Numerical Integrator (Time-Stepping) File" );
  if ( useStochastic )
    OpenFile( &stochasticFile, rootFileName, "_Stochastic.c",
              "The Stochastic Chemical Model File" );
  if ( useStoicmat ) {
    OpenFile( &stoichiomFile, rootFileName, "_Stoichiom.c",
              "The Stoichiometric Chemical Model File" );
    OpenFile( &sparse_stoicmFile, rootFileName, "_StoichiomSP.c",
              "Sparse Stoichiometric Data Structures File" );
  }
  OpenFile( &utilFile, rootFileName, "_Util.c", "Auxiliary Routines File" );
  OpenFile( &sparse_dataFile, rootFileName, "_Sparse.h", "Sparse Data Header File" );
  OpenFile( &global_dataFile, rootFileName, "_Global.h", "Global Data Header File" );
  OpenFile( &logFile, rootFileName, ".log", "Log File with Human-Readable Information" );
  OpenFile( &monitorFile, rootFileName, "_Monitor.c", "Utility Data Initialization" );
}
