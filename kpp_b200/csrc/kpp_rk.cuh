// Batched fully implicit Runge-Kutta integrator: the reference's C
// RungeKutta (int/runge_kutta.c: 3-stage Radau-2A, Lobatto-3C, Gauss,
// Radau-1A and the 4-stage Lobatto-3A, simplified Newton on the transformed
// system with one real and one complex sparse LU) for one cell per thread,
// on the generated Fun / Jac_SP / LU / solve device code and the complex LU
// of the mechanism's _cmplx header.  Included by kpp_rosenbrock.cu in its
// Runge-Kutta part (and in part 0, for the work layout).
//
// The arithmetic and the control flow are the reference's, operation for
// operation, including the behaviour of its C translation:
//  - RK_ErrorMsg only records the code: errors met while integrating (too
//    many steps, step too small, repeatedly singular matrix) are printed and
//    the integration goes on, and RK_Integrator ends with IERR = 1
//    (int/runge_kutta.c:701-1001); only the parameter checks of RungeKutta
//    return a negative IERR, the last failing check's code, before any step;
//  - ICNTRL[1] == 0 selects vector tolerances (ITOL = 1);
//  - ISTATUS counts only the Fun calls of the step start, the SDIRK error
//    estimate's Newton loop and the classic estimate's second solve; the
//    three stage evaluations of RK_PrepareRHS and the Lobatto-3A estimate's
//    evaluation are not counted; Nrej only after the first accepted step;
//  - RSTATUS[2] (Hnew) is recorded before the Hmin / Hmax clamp;
//  - Lobatto-3A runs through the 3-stage formulas with the upper-left 3x3
//    block of its 4x4 A (whose first row is zero).
// Two exits the reference does not have, for cells on which it would never
// return: H becoming 0 or NaN (IERR -10, the reference's "step size too
// small" code; there its loop runs forever) and more than Max_no_steps +
// kStepGrace steps (IERR -9; the reference prints -9 at Max_no_steps and
// continues, so every cell it finishes within that grace matches).
#pragma once

// Doubles of work storage one thread slot needs in the scratch layout: the
// Jacobian and the three LU factors (E1, E2R, E2I), 18 vectors, the complex
// LU's dense work row (two vectors, used by the generic form of large
// mechanisms), rate constants and the Fun / Jac_SP temporaries.
constexpr long kRkPerSlot = 4L * LU_NZ + 20L * NVAR + 2L * NREACT + KPP_NJAC_TMP;

namespace rk {

constexpr int kStepGrace = 200000;

// rkMethod codes of int/runge_kutta.c:26-30
enum { R2A = 1, R1A = 2, L3C = 3, GAU = 4, L3A = 5 };

// The coefficients the integrator reads, of one method
// (int/runge_kutta.c:1369-1996).
struct Method {
  int id;
  double A[3][3], C[3], D[3], E[4], Theta[3], F[3];
  double bgam0, bgam4, gamma, alpha, beta, elo;
  double T[3][3], TinvAinv[3][3];
};

// Everything RungeKutta derives from ICNTRL / RCNTRL that is the same for
// every cell; `ierr` is the last failing parameter check (0: none).
struct Controls {
  Method m;
  int ierr;
  bool vector_tol, sdirk_error, start_newton, gustafsson;
  int max_no_steps, newton_maxit;
  double theta_min, newton_tol, facsafe, facmin, facmax, facrej, qmin, qmax;
};

// The method tables, with the reference's expressions (computed on the
// host in IEEE double, as the reference computes them at run time).
inline void set_method(Method& m, int which, bool sdirk_error) {
  m = Method{};
  if (which == R2A) {
    const double b0 = sdirk_error ? (double)(0.2e-01) : (double)(0.5e-01);
    m.id = R2A;
    const double A[3][3] = {
        {1.968154772236604258683861429918299e-01, -6.55354258501983881085227825696087e-02,
         2.377097434822015242040823210718965e-02},
        {3.944243147390872769974116714584975e-01, 2.920734116652284630205027458970589e-01,
         -4.154875212599793019818600988496743e-02},
        {3.764030627004672750500754423692808e-01, 5.124858261884216138388134465196080e-01,
         1.111111111111111111111111111111111e-01}};
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) m.A[i][j] = A[i][j];
    m.C[0] = 1.550510257216821901802715925294109e-01;
    m.C[1] = 6.449489742783178098197284074705891e-01;
    m.C[2] = 1.0;
    m.D[0] = 0.0; m.D[1] = 0.0; m.D[2] = 1.0;
    m.E[0] = 1.0 * b0;
    m.E[1] = (-10.04880939982741556246032950764708) * b0;
    m.E[2] = 1.382142733160748895793662840980412 * b0;
    m.E[3] = (-.3333333333333333333333333333333333) * b0;
    m.bgam0 = b0;
    m.bgam4 = .2748888295956773677478286035994148;
    m.Theta[0] = (-1.520677486405081647234271944611547) - 10.04880939982741556246032950764708 * b0;
    m.Theta[1] = 2.070455145596436382729929151810376 + 1.382142733160748895793662840980413 * b0;
    m.Theta[2] = (-.3333333333333333333333333333333333) * b0 - .3744441479783868387391430179970741;
    m.elo = (b0 == 0.0) ? 6.0 : 4.0;
    m.gamma = 3.637834252744495732208418513577775;
    m.alpha = 2.681082873627752133895790743211112;
    m.beta = 3.050430199247410569426377624787569;
    const double T[3][3] = {
        {9.443876248897524148749007950641664e-02, -1.412552950209542084279903838077973e-01,
         -3.00291941051474244918611170890539e-02},
        {2.502131229653333113765090675125018e-01, 2.041293522937999319959908102983381e-01,
         3.829421127572619377954382335998733e-01},
        {1.0, 1.0, 0.0}};
    const double TIA[3][3] = {
        {1.520148562492775501049204957366528e+01, 1.192055789400527921212348994770778,
         1.903956760517560343018332287285119},
        {-9.669512977505946748632625374449567, -8.724028436822336183071773193986487,
         3.096043239482439656981667712714881},
        {-1.409513259499574544876303981551774e+01, 5.895975725255405108079130152868952,
         -1.441236197545344702389881889085515e-01}};
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) { m.T[i][j] = T[i][j]; m.TinvAinv[i][j] = TIA[i][j]; }
  } else if (which == L3C) {
    const double b0 = sdirk_error ? 0.2 : 0.5;
    m.id = L3C;
    const double A[3][3] = {
        {.1666666666666666666666666666666667, -.3333333333333333333333333333333333,
         .1666666666666666666666666666666667},
        {.1666666666666666666666666666666667, .4166666666666666666666666666666667,
         -.8333333333333333333333333333333333e-01},
        {.1666666666666666666666666666666667, .6666666666666666666666666666666667,
         .1666666666666666666666666666666667}};
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) m.A[i][j] = A[i][j];
    m.C[0] = 0.0; m.C[1] = 0.5; m.C[2] = 1.0;
    m.D[0] = 0.0; m.D[1] = 0.0; m.D[2] = 1.0;
    m.E[0] = .3808338772072650364017425226487022 * b0;
    m.E[1] = (-1.142501631621795109205227567946107) * b0;
    m.E[2] = (-1.523335508829060145606970090594809) * b0;
    m.E[3] = .3808338772072650364017425226487022 * b0;
    m.bgam0 = b0;
    m.bgam4 = .3808338772072650364017425226487021;
    m.Theta[0] = -3.0 * b0 - .3808338772072650364017425226487021;
    m.Theta[1] = -4.0 * b0 + 1.523335508829060145606970090594808;
    m.Theta[2] = (-.142501631621795109205227567946106) + b0;
    m.elo = (b0 == 0.0) ? 5.0 : 4.0;
    m.gamma = 2.625816818958466716011888933765284;
    m.alpha = 1.687091590520766641994055533117359;
    m.beta = 2.508731754924880510838743672432351;
    const double T[3][3] = {
        {1.0, 1.0, 0.0},
        {.4554100411010284672111720348287483, -.6027050205505142336055860174143743,
         -.4309321229203225731070721341350346},
        {2.195823345445647152832799205549709, -1.097911672722823576416399602774855,
         .7850032632435902184104551358922130}};
    const double TIA[3][3] = {
        {1.104302803159744452668648155627548, .916122120694355522658740710823143,
         .5029105849749601702795812241441172},
        {1.895697196840255547331351844372453, 3.083877879305644477341259289176857,
         -1.502910584974960170279581224144117},
        {.8362439183082935036129145574774502, -3.344975673233174014451658229909802,
         .312908409479233358005944466882642}};
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) { m.T[i][j] = T[i][j]; m.TinvAinv[i][j] = TIA[i][j]; }
  } else if (which == GAU) {
    const double b0 = 0.1;
    m.id = GAU;
    const double A[3][3] = {
        {.1388888888888888888888888888888889, -.359766675249389034563954710966045e-01,
         .97894440153083260495800422294756e-02},
        {.3002631949808645924380249472131556, .2222222222222222222222222222222222,
         -.224854172030868146602471694353778e-01},
        {.2679883337624694517281977355483022, .4804211119693833479008399155410489,
         .1388888888888888888888888888888889}};
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) m.A[i][j] = A[i][j];
    m.C[0] = .1127016653792583114820734600217600;
    m.C[1] = .5000000000000000000000000000000000;
    m.C[2] = .8872983346207416885179265399782400;
    m.D[0] = .1666666666666666666666666666666667e+01;
    m.D[1] = -.1333333333333333333333333333333333e+01;
    m.D[2] = .1666666666666666666666666666666667e+01;
    m.E[0] = .2153144231161121782447335303806954 * b0;
    m.E[1] = (-2.825278112319014084275808340593191) * b0;
    m.E[2] = .2870858974881495709929780405075939 * b0;
    m.E[3] = (-.4558086256248162565397206448274867e-01) * b0;
    m.bgam0 = 0.0;
    m.bgam4 = .2153144231161121782447335303806955;
    m.Theta[0] = -2.594040933093095272574031876464493;
    m.Theta[1] = 1.824611539036311947589425112250199;
    m.Theta[2] = .1856563166634371860478043996459493;
    m.elo = 4.0;
    m.gamma = 4.644370709252171185822941421408064;
    m.alpha = 3.677814645373914407088529289295970;
    m.beta = 3.508761919567443321903661209182446;
    const double T[3][3] = {
        {.7215185205520017032081769924397664e-01, -.8224123057363067064866206597516454e-01,
         -.6012073861930850173085948921439054e-01},
        {.1188325787412778070708888193730294, .5306509074206139504614411373957448e-01,
         .3162050511322915732224862926182701},
        {1.0, 1.0, 0.0}};
    const double TIA[3][3] = {
        {27.82766708436744962047620566703329, 5.290933503982655311815946575100597,
         2.007817718512643701322151051660114},
        {-17.66368928942422710690385180065675, -14.45491129892587782538830044147713,
         2.992182281487356298677848948339886},
        {-25.60678350282974256072419392007303, 6.762434375611708328910623303779923,
         1.043979339483109825041215970036771}};
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) { m.T[i][j] = T[i][j]; m.TinvAinv[i][j] = TIA[i][j]; }
  } else if (which == R1A) {
    const double b0 = 0.1;
    m.id = R1A;
    const double A[3][3] = {
        {.1111111111111111111111111111111111, -.1916383190435098943442935597058829,
         .8052720793239878323318244859477174e-01},
        {.1111111111111111111111111111111111, .2920734116652284630205027458970589,
         -.481334970546573839513422644787591e-01},
        {.1111111111111111111111111111111111, .5370223859435462728402311533676479,
         .1968154772236604258683861429918299}};
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) m.A[i][j] = A[i][j];
    m.C[0] = 0.0;
    m.C[1] = .3550510257216821901802715925294109;
    m.C[2] = .8449489742783178098197284074705891;
    m.D[0] = .3333333333333333333333333333333333;
    m.D[1] = -.8914115380582557157653087040196127;
    m.D[2] = 1.558078204724922382431975370686279;
    m.E[0] = .2748888295956773677478286035994148 * b0;
    m.E[1] = (-1.374444147978386838739143017997074) * b0;
    m.E[2] = (-1.335337922441686804550326197041126) * b0;
    m.E[3] = .235782604058977333559011782643466 * b0;
    m.bgam0 = 0.0;
    m.bgam4 = .2748888295956773677478286035994148;
    m.Theta[0] = -1.224370034375505083904362087063351;
    m.Theta[1] = .9340045331532641409047527962010133;
    m.Theta[2] = .4656990124352088397561234800640929;
    m.elo = 4.0;
    m.gamma = 3.637834252744495732208418513577775;
    m.alpha = 2.681082873627752133895790743211112;
    m.beta = 3.050430199247410569426377624787569;
    const double T[3][3] = {
        {.424293819848497965354371036408369, -.3235571519651980681202894497035503,
         -.522137786846287839586599927945048},
        {.57594609499806128896291585429339e-01, .3148663231849760131614374283783e-02,
         .452429247674359778577728510381731},
        {1.0, 1.0, 0.0}};
    const double TIA[3][3] = {
        {4.487354449794728738538663081025420, 5.178748573958397475446442544234494,
         1.435609490412123627047824222335563},
        {-2.854361287939276673073807031221493, -1.003648660720543859000994063139137e+01,
         1.789135380979465422050817815017383},
        {-4.160768067752685525282947313530352, 1.124128569859216916690209918405860,
         1.700644430961823796581896350418417}};
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) { m.T[i][j] = T[i][j]; m.TinvAinv[i][j] = TIA[i][j]; }
  } else if (which == L3A) {
    m.id = L3A;
    // the upper-left 3x3 block of the 4-stage A, as the 3-stage formulas read it
    const double A[3][3] = {
        {0.0, 0.0, 0.0},
        {.11030056647916491413674311390609397, .1896994335208350858632568860939060,
         -.339073642291438837776604807792215e-01},
        {.73032766854168419196590219427239365e-01, .4505740308958105504443271474458881,
         .2269672331458315808034097805727606}};
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) m.A[i][j] = A[i][j];
    m.C[0] = 0.0;
    m.C[1] = .2763932022500210303590826331268724;
    m.C[2] = .7236067977499789696409173668731276;
    m.D[0] = 0.0; m.D[1] = 0.0; m.D[2] = 0.0;
    m.E[0] = .1957403846510110711315759367097231e-01;
    m.E[1] = -.1986820345632580910316020806676438;
    m.E[2] = .1660586371214229125096727578826900;
    m.E[3] = -.9787019232550553556578796835486154e-01;
    m.F[0] = 0.0;
    m.F[1] = -.66535815876916686607437314126436349;
    m.F[2] = 1.7419302743497277572980407931678409;
    m.elo = 4.0;
    m.bgam0 = .2950472755430528877214995073815946e-01;
    m.bgam4 = .2153144231161121782447335303806956;
    m.Theta[0] = 0.0;
    m.Theta[1] = -.6653581587691668660743731412643631;
    m.Theta[2] = 1.741930274349727757298040793167842;
    m.gamma = 4.644370709252171185822941421408063;
    m.alpha = 3.677814645373914407088529289295968;
    m.beta = 3.508761919567443321903661209182446;
    const double T[3][3] = {
        {.5303036326129938105898786144870856e-01, -.7776129960563076320631956091016914e-01,
         .6043307469475508514468017399717112e-02},
        {.2637242522173698467283726114649606, .2193839918662961493126393244533346,
         .3198765142300936188514264752235344},
        {1.0, 0.0, 0.0}};
    const double TIA[3][3] = {
        {35.73858579417120341641749040405149, -.675195748578927863668368190236025,
         2.927206016036483646751158874041632},
        {-24.55824590667225493437162206039511, -10.50514413892002061837750015342036,
         4.072793983963516353248841125958369},
        {-30.92301972744621647251975054630589, 12.08182467154052413351908559269928,
         -1.546411207640594954081233702132946}};
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) { m.T[i][j] = T[i][j]; m.TinvAinv[i][j] = TIA[i][j]; }
  }
}

// RungeKutta's parameter handling (int/runge_kutta.c:270-603) for the
// controls every cell shares; Hmin / Hmax / Hstart (per cell, through
// |Tend - T|) and the tolerance check (device arrays) are done per cell.
inline Controls make_controls(const int* icntrl, const double* rcntrl) {
  Controls c{};
  c.ierr = 0;
  c.vector_tol = icntrl[1] == 0;
  c.sdirk_error = icntrl[9] != 0;
  switch (icntrl[2]) {
    case 0:
    case 1: set_method(c.m, R2A, c.sdirk_error); break;
    case 2: set_method(c.m, L3C, c.sdirk_error); break;
    case 3: set_method(c.m, GAU, c.sdirk_error); break;
    case 4: set_method(c.m, R1A, c.sdirk_error); break;
    case 5: set_method(c.m, L3A, c.sdirk_error); break;
    default: c.ierr = -13;
  }
  if (icntrl[3] == 0) {
    c.max_no_steps = 200000;
  } else {
    c.max_no_steps = icntrl[3];
    if (c.max_no_steps <= 0) c.ierr = -1;
  }
  if (icntrl[4] == 0) {
    c.newton_maxit = 8;
  } else {
    c.newton_maxit = icntrl[4];
    if (c.newton_maxit <= 0) c.ierr = -2;
  }
  c.start_newton = icntrl[5] == 0;
  c.gustafsson = icntrl[10] == 0;
  const double roundoff = kRoundoff;
  c.facmin = rcntrl[3] == 0.0 ? 0.2 : rcntrl[3];
  c.facmax = rcntrl[4] == 0.0 ? 8.0 : rcntrl[4];
  c.facrej = rcntrl[5] == 0.0 ? 0.1 : rcntrl[5];
  c.facsafe = rcntrl[6] == 0.0 ? 0.9 : rcntrl[6];
  if ((c.facmax < 1.0) || (c.facmin > 1.0) || (c.facsafe <= 1.0e-03) || (c.facsafe >= 1.0))
    c.ierr = -4;
  if (rcntrl[7] == 0.0) {
    c.theta_min = 1.0e-03;
  } else {
    c.theta_min = rcntrl[7];
    if (c.theta_min <= 0.0 || c.theta_min >= 1.0) c.ierr = -5;
  }
  if (rcntrl[8] == 0.0) {
    c.newton_tol = 3.0e-02;
  } else {
    c.newton_tol = rcntrl[8];
    if (c.newton_tol <= roundoff) c.ierr = -6;
  }
  c.qmin = rcntrl[9] == 0.0 ? 1.0 : rcntrl[9];
  c.qmax = rcntrl[10] == 0.0 ? 1.2 : rcntrl[10];
  if (c.qmin > 1.0 || c.qmax < 1.0) c.ierr = -7;
  return c;
}

#if !defined(KPP_RK_HOST_ONLY)

// Per-cell work arrays: the Jacobian (kept for SkipJac), the real LU E1 and
// the complex LU (E2R, E2I); Y, FO, SCAL, Z1..Z4, DZ1..DZ4, G, TMP, the
// stage value F, the estimate's F2 and the interpolation polynomial CONT;
// the complex LU's work row (WR, WI); rate constants and the Fun / Jac_SP
// temporaries.
constexpr long kPerSlot = kRkPerSlot;

#if defined(KPP_SCRATCH)
struct Work {
  Strided y, fo, scal, z1, z2, z3, z4, dz1, dz2, dz3, dz4, g, tmp, f, f2, c0, c1, c2, wr, wi;
  Strided fjac, e1, e2r, e2i, rconst, a, b;
  __device__ __forceinline__ Work(double* base, long slot) {
    double* block = base + (slot / kLanes) * kPerSlot * kLanes + (slot % kLanes);
    long off = 0;
    auto take = [&](long n) {
      Strided v{block + off * kLanes};
      off += n;
      return v;
    };
    y = take(NVAR); fo = take(NVAR); scal = take(NVAR);
    z1 = take(NVAR); z2 = take(NVAR); z3 = take(NVAR); z4 = take(NVAR);
    dz1 = take(NVAR); dz2 = take(NVAR); dz3 = take(NVAR); dz4 = take(NVAR);
    g = take(NVAR); tmp = take(NVAR); f = take(NVAR); f2 = take(NVAR);
    c0 = take(NVAR); c1 = take(NVAR); c2 = take(NVAR); wr = take(NVAR); wi = take(NVAR);
    fjac = take(LU_NZ); e1 = take(LU_NZ); e2r = take(LU_NZ); e2i = take(LU_NZ);
    rconst = take(NREACT); a = take(NREACT); b = take(KPP_NJAC_TMP);
  }
};
#else
struct Work {
  double y[NVAR], fo[NVAR], scal[NVAR], z1[NVAR], z2[NVAR], z3[NVAR], z4[NVAR];
  double dz1[NVAR], dz2[NVAR], dz3[NVAR], dz4[NVAR], g[NVAR], tmp[NVAR], f[NVAR], f2[NVAR];
  double c0[NVAR], c1[NVAR], c2[NVAR], wr[NVAR], wi[NVAR];
  double fjac[LU_NZ], e1[LU_NZ], e2r[LU_NZ], e2i[LU_NZ];
  double rconst[NREACT > 0 ? NREACT : 1], a[NREACT > 0 ? NREACT : 1], b[KPP_NJAC_TMP];
  __device__ __forceinline__ Work(double*, long) {}
};
#endif

// SIGN(x, y) of int/runge_kutta.c:7, with the ABS macro of :4
__device__ __forceinline__ double rk_sign(double x, double y) {
  return (y >= 0) ? ros_abs(x) : -ros_abs(x);
}

template <class TX>
__device__ __forceinline__ void zero(TX& x) {
#pragma unroll 4
  for (int i = 0; i < NVAR; i++) x[i] = 0.0;
}

// RK_ErrorScale (int/runge_kutta.c:1063-1082)
template <class W>
__device__ __forceinline__ void error_scale(W& w, const double* atol, const double* rtol,
                                            bool vector_tol) {
#pragma unroll 4
  for (int i = 0; i < NVAR; i++) {
    const double a = vector_tol ? atol[i] : atol[0], r = vector_tol ? rtol[i] : rtol[0];
    w.scal[i] = 1.0 / (a + r * ros_abs(w.y[i]));
  }
}

// RK_ErrorNorm (int/runge_kutta.c:1355-1366): sqrt(mean((dy scal)^2)), at
// least 1e-10; the reference's SQRT is pow(x, 0.5), computed here as the
// correctly rounded sqrt.
template <class TD, class TS>
__device__ __forceinline__ double error_norm(const TD& dy, const TS& scal) {
  double e = 0.0;
#pragma unroll 4
  for (int i = 0; i < NVAR; i++) e = e + (dy[i] * scal[i]) * (dy[i] * scal[i]);
  const double r = sqrt(e / (double)NVAR);
  return r >= 1.0e-10 ? r : 1.0e-10;
}

// FUN_CHEM(T, V, F) (int/runge_kutta.c:1997-2010): rates at T, then Fun.
template <class W, class TV, class TF>
__device__ __forceinline__ void fun_chem(const CellEnv& env, double t, const TV& v, TF& f, W& w) {
  if (rates_vary<W>(env)) rates_at(env, t, w);
  kpp_fun(v, env.fix, w.rconst, f, w.a);
}

// RK_Interpolate "make" (int/runge_kutta.c:1108-1131)
template <class W>
__device__ __forceinline__ void interpolate_make(const Method& m, W& w) {
  const double* C = m.C;
  const double den = (C[2] - C[1]) * (C[1] - C[0]) * (C[0] - C[2]);
#pragma unroll 2
  for (int i = 0; i < NVAR; i++) {
    const double Z1 = w.z1[i], Z2 = w.z2[i], Z3 = w.z3[i];
    w.c0[i] = (-C[2] * C[2] * C[1] * Z1 + Z3 * C[1] * C[0] * C[0] + C[1] * C[1] * C[2] * Z1 -
               C[1] * C[1] * C[0] * Z3 + C[2] * C[2] * C[0] * Z2 - Z2 * C[2] * C[0] * C[0]) /
                  den -
              Z3;
    w.c1[i] = -(C[0] * C[0] * (Z3 - Z2) + C[1] * C[1] * (Z1 - Z3) + C[2] * C[2] * (Z2 - Z1)) / den;
    w.c2[i] = (C[0] * (Z3 - Z2) + C[1] * (Z1 - Z3) + C[2] * (Z2 - Z1)) / den;
  }
}

// RK_Interpolate "eval" (int/runge_kutta.c:1132-1145)
template <class W>
__device__ __forceinline__ void interpolate_eval(const Method& m, double h, double hold, W& w) {
  const double r = h / hold;
  const double x1 = 1.0 + m.C[0] * r, x2 = 1.0 + m.C[1] * r, x3 = 1.0 + m.C[2] * r;
#pragma unroll 2
  for (int i = 0; i < NVAR; i++) {
    const double c0 = w.c0[i], c1 = w.c1[i], c2 = w.c2[i];
    w.z1[i] = c0 + x1 * (c1 + x1 * c2);
    w.z2[i] = c0 + x2 * (c1 + x2 * c2);
    w.z3[i] = c0 + x3 * (c1 + x3 * c2);
  }
}

// RK_PrepareRHS (int/runge_kutta.c:1152-1187): DZ_i = Z_i - h sum_j A_ij F(Y + Z_j)
template <class W>
__device__ __forceinline__ void prepare_rhs(const CellEnv& env, const Method& m, double t,
                                            double h, W& w) {
  copy(w.z1, w.dz1);
  copy(w.z2, w.dz2);
  copy(w.z3, w.dz3);
  if (m.id == L3A) {
    axpy(-h * m.A[0][0], w.fo, w.dz1);
    axpy(-h * m.A[1][0], w.fo, w.dz2);
    axpy(-h * m.A[2][0], w.fo, w.dz3);
  }
#pragma unroll 4
  for (int i = 0; i < NVAR; i++) w.tmp[i] = w.y[i] + w.z1[i];
  fun_chem(env, t + m.C[0] * h, w.tmp, w.f, w);
  axpy(-h * m.A[0][0], w.f, w.dz1);
  axpy(-h * m.A[1][0], w.f, w.dz2);
  axpy(-h * m.A[2][0], w.f, w.dz3);
#pragma unroll 4
  for (int i = 0; i < NVAR; i++) w.tmp[i] = w.y[i] + w.z2[i];
  fun_chem(env, t + m.C[1] * h, w.tmp, w.f, w);
  axpy(-h * m.A[0][1], w.f, w.dz1);
  axpy(-h * m.A[1][1], w.f, w.dz2);
  axpy(-h * m.A[2][1], w.f, w.dz3);
#pragma unroll 4
  for (int i = 0; i < NVAR; i++) w.tmp[i] = w.y[i] + w.z3[i];
  fun_chem(env, t + m.C[2] * h, w.tmp, w.f, w);
  axpy(-h * m.A[0][2], w.f, w.dz1);
  axpy(-h * m.A[1][2], w.f, w.dz2);
  axpy(-h * m.A[2][2], w.f, w.dz3);
}

// RK_Decomp (int/runge_kutta.c:1190-1246): E1 = gamma/h - J (real LU) and
// E2 = (alpha + i beta)/h - J (complex LU); returns the singular row or 0.
template <class W>
__device__ __forceinline__ int decomp(const Method& m, double h, W& w, Stats& st) {
  const double gamma_h = m.gamma / h, alpha_h = m.alpha / h, beta_h = m.beta / h;
#pragma unroll 4
  for (int i = 0; i < LU_NZ; i++) w.e1[i] = -w.fjac[i];
  kpp_add_diagonal(w.e1, gamma_h);
  int ising = kpp_decomp(w.e1, w.wr);  // wr: the complex LU's work row, free here
  if (ising != 0) {
    st.ndec++;
    return ising;
  }
#pragma unroll 4
  for (int i = 0; i < LU_NZ; i++) {
    w.e2r[i] = -w.fjac[i];
    w.e2i[i] = 0.0;
  }
  kpp_add_diagonal(w.e2r, alpha_h);
  kpp_add_diagonal(w.e2i, beta_h);
#if defined(KPP_CMPLX_GENERIC)
  ising = kpp_decomp_cmplx_w(w.e2r, w.e2i, w.wr, w.wi);
#else
  ising = kpp_decomp_cmplx(w.e2r, w.e2i);
#endif
  st.ndec++;
  return ising;
}

// RK_Solve (int/runge_kutta.c:1249-1295) on DZ1..DZ3: transform with
// Tinv Ainv / h, the real solve for the first component, the complex solve
// for the pair, back-transform with T.
template <class W>
__device__ __forceinline__ void solve(const Method& m, double h, W& w, Stats& st) {
#pragma unroll 2
  for (int i = 0; i < NVAR; i++) {
    const double x1 = w.dz1[i] / h, x2 = w.dz2[i] / h, x3 = w.dz3[i] / h;
    w.dz1[i] = m.TinvAinv[0][0] * x1 + m.TinvAinv[0][1] * x2 + m.TinvAinv[0][2] * x3;
    w.dz2[i] = m.TinvAinv[1][0] * x1 + m.TinvAinv[1][1] * x2 + m.TinvAinv[1][2] * x3;
    w.dz3[i] = m.TinvAinv[2][0] * x1 + m.TinvAinv[2][1] * x2 + m.TinvAinv[2][2] * x3;
  }
  kpp_solve(w.e1, w.dz1);
  kpp_solve_cmplx(w.e2r, w.e2i, w.dz2, w.dz3);
#pragma unroll 2
  for (int i = 0; i < NVAR; i++) {
    const double x1 = w.dz1[i], x2 = w.dz2[i], x3 = w.dz3[i];
    w.dz1[i] = m.T[0][0] * x1 + m.T[0][1] * x2 + m.T[0][2] * x3;
    w.dz2[i] = m.T[1][0] * x1 + m.T[1][1] * x2 + m.T[1][2] * x3;
    w.dz3[i] = m.T[2][0] * x1 + m.T[2][1] * x2 + m.T[2][2] * x3;
  }
  st.nsol++;
}

// RK_ErrorEstimate (int/runge_kutta.c:1298-1352), the classic estimator.
template <class W>
__device__ __forceinline__ double error_estimate(const CellEnv& env, const Method& m, double h,
                                                 double t, bool first_step, bool reject, W& w,
                                                 Stats& st) {
  const double hrk_e1 = m.E[1] / h, hrk_e2 = m.E[2] / h, hrk_e3 = m.E[3] / h;
#pragma unroll 4
  for (int i = 0; i < NVAR; i++) {
    w.f2[i] = hrk_e1 * w.z1[i] + hrk_e2 * w.z2[i] + hrk_e3 * w.z3[i];
    w.tmp[i] = m.E[0] * w.fo[i] + w.f2[i];
  }
  kpp_solve(w.e1, w.tmp);
  if ((m.id == R1A) || (m.id == GAU) || (m.id == L3A)) kpp_solve(w.e1, w.tmp);
  if (m.id == GAU) kpp_solve(w.e1, w.tmp);
  double err = error_norm(w.tmp, w.scal);
  if (err < 1.0) return err;
  if (first_step || reject) {
#pragma unroll 4
    for (int i = 0; i < NVAR; i++) w.tmp[i] = w.y[i] + w.tmp[i];
    fun_chem(env, t, w.tmp, w.f, w);  // F1
    st.nfun++;
#pragma unroll 4
    for (int i = 0; i < NVAR; i++) w.tmp[i] = w.f[i] + w.f2[i];
    kpp_solve(w.e1, w.tmp);
    err = error_norm(w.tmp, w.scal);
  }
  return err;
}

// The SDIRK error estimator's Newton loop (int/runge_kutta.c:836-887);
// returns whether it converged, `fac` the step factor when it did not.
template <class W>
__device__ __forceinline__ bool sdirk_newton(const CellEnv& env, const Controls& c, double t,
                                             double h, double& fac, W& w, Stats& st) {
  const Method& m = c.m;
  copy(w.z3, w.z4);
  zero(w.g);
  if (m.id != L3A) axpy(m.bgam0 * h, w.fo, w.g);
  axpy(m.Theta[0], w.z1, w.g);
  axpy(m.Theta[1], w.z2, w.g);
  axpy(m.Theta[2], w.z3, w.g);
  bool done = false;
  fac = 0.5;
  double rate = 2.0, inc_old = 0.0;
  for (int it = 1; it <= c.newton_maxit; it++) {
#pragma unroll 4
    for (int i = 0; i < NVAR; i++) w.tmp[i] = w.y[i] + w.z4[i];
    fun_chem(env, t + h, w.tmp, w.dz4, w);
    st.nfun++;
    axpy(-1.0 * m.gamma / h, w.z4, w.dz4);
    axpy(m.gamma / h, w.g, w.dz4);
    kpp_solve(w.e1, w.dz4);
    const double inc = error_norm(w.dz4, w.scal);
    if (it == 1) {
      rate = 2.0;
    } else {
      const double theta_sd = inc / inc_old;
      if (theta_sd < 0.99) {
        rate = theta_sd / (1.0 - theta_sd);
        const double predicted =
            inc * KPP_POW(theta_sd, (double)(c.newton_maxit - it)) / (1.0 - theta_sd);
        if (predicted >= c.newton_tol) {
          const double qn = ros_min(10.0, predicted / c.newton_tol);
          fac = 0.8 * KPP_POW(qn, (-1.0 / (double)(1 + c.newton_maxit - it)));
          break;
        }
      } else {
        break;
      }
    }
    inc_old = inc;
    axpy(1.0, w.dz4, w.z4);
    done = (rate * inc <= c.newton_tol);
    if (done) break;
  }
  return done;
}

// RK_Integrator (int/runge_kutta.c:616-1001) for one cell.  Returns 1, or
// -10 / -9 at the two exits of the header comment.
template <class W>
__device__ int integrate(const CellEnv& env, W& w, const Controls& c, double t, double tend,
                         double hmin, double hmax, double hstart, const double* atol,
                         const double* rtol, double rst[3], Stats& st) {
  const Method& m = c.m;
  const double roundoff = kRoundoff;
  double hacc = 0.0, errold = 0.0;
  const double tdir = rk_sign(1.0, tend - t);
  double h = ros_min(ros_max(ros_abs(hmin), ros_abs(hstart)), hmax);
  if (ros_abs(h) <= 10.0 * roundoff) h = 1.0e-06;
  h = rk_sign(h, tdir);
  double hold = h;
  bool reject = false, first_step = true, skip_jac = false, skip_lu = false;
  if ((t + h * 1.0001 - tend) * tdir >= 0.0) h = tend - t;
  double theta = 0.0;
  rates_once(env, t, w);
  error_scale(w, atol, rtol, c.vector_tol);

  while ((tend - t) * tdir - roundoff > 0.0) {
    if (h == 0.0 || h != h) return -10;  // the reference would loop here for ever
    fun_chem(env, t, w.y, w.fo, w);      // FUN_CHEM(T, Y, FO)
    st.nfun++;
    if (!skip_lu) {
      if (!skip_jac) {  // JAC_CHEM(T, Y, FJAC): the rates at T are in place
        kpp_jac_sp<false>(w.y, env.fix, w.rconst, w.fjac, w.b);
        st.njac++;
      }
      if (decomp(m, h, w, st) != 0) {
        st.nsng++;  // five in a row: the reference prints -12 and goes on
        h = h * 0.5;
        reject = true;
        skip_jac = true;
        skip_lu = false;
        continue;
      }
    }
    st.nstp++;
    if (st.nstp > c.max_no_steps + kStepGrace) return -9;
    // (the reference prints -9 beyond Max_no_steps and -10 when 0.1|H| <=
    // |T| Roundoff, and goes on)
    if (first_step || !c.start_newton) {
      zero(w.z1);
      zero(w.z2);
      zero(w.z3);
    } else {
      interpolate_eval(m, h, hold, w);
    }
    bool done = false;
    double fac = 0.5, rate = 2.0, inc_old = 0.0;
    int it;
    for (it = 1; it <= c.newton_maxit; it++) {
      prepare_rhs(env, m, t, h, w);
      solve(m, h, w, st);
      const double n1 = error_norm(w.dz1, w.scal), n2 = error_norm(w.dz2, w.scal),
                   n3 = error_norm(w.dz3, w.scal);
      const double inc = sqrt((n1 * n1 + n2 * n2 + n3 * n3) / 3.0);
      if (it == 1) {
        theta = ros_abs(c.theta_min);
        rate = 2.0;
      } else {
        theta = inc / inc_old;
        if (theta < 0.99) {
          rate = theta / (1.0 - theta);
        } else {
          break;
        }
        if (it < c.newton_maxit) {
          const double predicted =
              inc * KPP_POW(theta, (double)(c.newton_maxit - it)) / (1.0 - theta);
          if (predicted >= c.newton_tol) {
            const double qn = ros_min(10.0, predicted / c.newton_tol);
            fac = 0.8 * KPP_POW(qn, (-1.0 / (double)(1 + c.newton_maxit - it)));
            break;
          }
        }
      }
      inc_old = ros_max(inc, roundoff);
      axpy(-1.0, w.dz1, w.z1);
      axpy(-1.0, w.dz2, w.z2);
      axpy(-1.0, w.dz3, w.z3);
      done = (rate * inc <= c.newton_tol);
      if (done) break;
    }
    const int it_main = it;
    if (!done) {
      h = fac * h;
      reject = true;
      skip_jac = true;
      skip_lu = false;
      continue;
    }

    double err;
    if (c.sdirk_error) {
      if (!sdirk_newton(env, c, t, h, fac, w, st)) {
        h = fac * h;
        reject = true;
        skip_jac = true;
        skip_lu = false;
        continue;
      }
      zero(w.dz4);
      if (m.id == L3A) {
#pragma unroll 4
        for (int i = 0; i < NVAR; i++) w.dz4[i] = h * m.F[0] * w.fo[i];
        if (m.F[0] != 0.0) axpy(m.F[0], w.z1, w.dz4);
        if (m.F[1] != 0.0) axpy(m.F[1], w.z2, w.dz4);
        if (m.F[2] != 0.0) axpy(m.F[2], w.z3, w.dz4);
#pragma unroll 4
        for (int i = 0; i < NVAR; i++) w.tmp[i] = w.y[i] + w.z4[i];
        fun_chem(env, t + h, w.tmp, w.dz1, w);
        axpy(h * m.bgam4, w.dz1, w.dz4);
      } else {
        if (m.D[0] != 0.0) axpy(m.D[0], w.z1, w.dz4);
        if (m.D[1] != 0.0) axpy(m.D[1], w.z2, w.dz4);
        if (m.D[2] != 0.0) axpy(m.D[2], w.z3, w.dz4);
        axpy(-1.0, w.z4, w.dz4);
      }
      err = error_norm(w.dz4, w.scal);
    } else {
      err = error_estimate(env, m, h, t, first_step, reject, w, st);
    }

    // new step size (the main loop's Newton count)
    fac = KPP_POW(err, (-1.0 / m.elo)) *
          ros_min(c.facsafe,
                  (1.0 + 2 * c.newton_maxit) / (double)(it_main + 2 * c.newton_maxit));
    fac = ros_min(c.facmax, ros_max(c.facmin, fac));
    double hnew = fac * h;
    if (err < 1.0) {  // accept
      first_step = false;
      st.nacc++;
      if (c.gustafsson) {
        if (st.nacc > 1) {
          double facgus = c.facsafe * (h / hacc) * KPP_POW(err * err / errold, -0.25);
          facgus = ros_min(c.facmax, ros_max(c.facmin, facgus));
          fac = ros_min(fac, facgus);
          hnew = fac * h;
        }
        hacc = h;
        errold = ros_max(1.0e-02, err);
      }
      hold = h;
      t = t + h;
      if (m.D[0] != 0.0) axpy(m.D[0], w.z1, w.y);
      if (m.D[1] != 0.0) axpy(m.D[1], w.z2, w.y);
      if (m.D[2] != 0.0) axpy(m.D[2], w.z3, w.y);
      if (c.start_newton) interpolate_make(m, w);
      error_scale(w, atol, rtol, c.vector_tol);
      rst[0] = t;
      rst[2] = hnew;
      rst[1] = h;
      hnew = tdir * ros_min(ros_max(ros_abs(hnew), hmin), hmax);
      if (reject) hnew = tdir * ros_min(ros_abs(hnew), ros_abs(h));
      reject = false;
      if ((t + hnew / c.qmin - tend) * tdir >= 0.0) {
        h = tend - t;
      } else {
        const double hratio = hnew / h;
        skip_lu = (theta <= c.theta_min) && (hratio >= c.qmin) && (hratio <= c.qmax);
        if (!skip_lu) h = hnew;
      }
      skip_jac = false;
    } else {  // reject
      if (first_step || reject)
        h = c.facrej * h;
      else
        h = hnew;
      reject = true;
      skip_jac = true;
      skip_lu = false;
      if (st.nacc >= 1) st.nrej++;
    }
  }
  return 1;
}

// RungeKutta for one cell (int/runge_kutta.c:203-603): the per-cell step
// bounds and the tolerance check, then the integrator; `c.ierr` < 0 (a
// failed shared parameter check) returns before any step, as does a failed
// tolerance check (-8, the last check).
template <class W>
__device__ int rk_cell(const CellEnv& env, W& w, const Controls& c, double t, double tend,
                       const double* rcntrl, const double* atol, const double* rtol,
                       double rst[3], Stats& st) {
  int ierr = c.ierr;
  const double roundoff = kRoundoff;
  if (!c.vector_tol) {
    if (atol[0] <= 0.0 || rtol[0] <= (10.0 * roundoff)) ierr = -8;
  } else {
    for (int i = 0; i < NVAR; i++)
      if ((atol[i] <= 0.0) || (rtol[i] <= 10.0 * roundoff)) ierr = -8;
  }
  if (ierr < 0) return ierr;
  const double span = ros_abs_diff(tend, t);
  const double hmin = rcntrl[0] == 0.0 ? 0.0 : ros_min(ros_abs(rcntrl[0]), span);
  const double hmax = rcntrl[1] == 0.0 ? span : ros_min(ros_abs(rcntrl[1]), span);
  const double hstart = rcntrl[2] == 0.0 ? 0.0 : ros_min(ros_abs(rcntrl[2]), span);
  return integrate(env, w, c, t, tend, hmin, hmax, hstart, atol, rtol, rst, st);
}

#endif  // !KPP_RK_HOST_ONLY

}  // namespace rk
