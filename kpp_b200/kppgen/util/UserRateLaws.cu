// kpp_b200 CUDA target of the KPP generator: the rate-law template pasted
// into <root>_Rates.cu (the C target pastes util/UserRateLaws.c there).
//
// The rate laws of util/UserRateLaws.c (Arrhenius forms, EP2, EP3, FALL) are
// the device functions of kpp_b200's kpp_ratelaws.cuh, which keep the C
// routines' single-precision argument rounding; these macros bind them to the
// TEMP and CFACTOR arguments of the device Update_RCONST.
#include "kpp_ratelaws.cuh"
#define ARR_abc(a0, b0, c0) kpp_arr_abc(TEMP, (float)(a0), (float)(b0), (float)(c0))
#define ARR_ab(a0, b0) kpp_arr_ab(TEMP, (float)(a0), (float)(b0))
#define ARR_ac(a0, c0) kpp_arr_ac(TEMP, (float)(a0), (float)(c0))
#define EP2(a0, c0, a2, c2, a3, c3) \
  kpp_ep2(TEMP, CFACTOR, (float)(a0), (float)(c0), (float)(a2), (float)(c2), (float)(a3), (float)(c3))
#define EP3(a1, c1, a2, c2) \
  kpp_ep3(TEMP, CFACTOR, (float)(a1), (float)(c1), (float)(a2), (float)(c2))
#define FALL(a0, b0, c0, a1, b1, c1, cf)                                                   \
  kpp_fall(TEMP, CFACTOR, (float)(a0), (float)(b0), (float)(c0), (float)(a1), (float)(b1), \
           (float)(c1), (float)(cf))
