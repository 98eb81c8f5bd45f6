// Device versions of the KPP utility templates used inside the rate
// constants: the rate-law functions of util/UserRateLaws.c:9-78 and the
// diurnal sun function of util/UpdateSun.c:1-20.
//
// The reference declares the rate-law arguments `float` (the mechanism's
// numbers are single precision by KPP convention) and computes in double; the
// generated code converts every argument to float before the call, so these
// take float and widen exactly where the reference does.  The order of the
// double operations is the reference's.
#pragma once

__device__ __forceinline__ double kpp_arr_abc(double TEMP, float A0, float B0, float C0) {
  return (double)A0 * exp(-(double)B0 / TEMP) * pow((TEMP / 300.0), (double)C0);
}

__device__ __forceinline__ double kpp_arr_ab(double TEMP, float A0, float B0) {
  return (double)A0 * exp(-(double)B0 / TEMP);
}

__device__ __forceinline__ double kpp_arr_ac(double TEMP, float A0, float C0) {
  return (double)A0 * pow((TEMP / 300.0), (double)C0);
}

__device__ __forceinline__ double kpp_ep2(double TEMP, double CFACTOR, float A0, float C0,
                                          float A2, float C2, float A3, float C3) {
  double K0 = (double)A0 * exp(-(double)C0 / TEMP);
  double K2 = (double)A2 * exp(-(double)C2 / TEMP);
  double K3 = (double)A3 * exp(-(double)C3 / TEMP);
  K3 = K3 * CFACTOR * 1.0e+6;
  return K0 + K3 / (1.0 + K3 / K2);
}

__device__ __forceinline__ double kpp_ep3(double TEMP, double CFACTOR, float A1, float C1,
                                          float A2, float C2) {
  double K1 = (double)A1 * exp(-(double)C1 / TEMP);
  double K2 = (double)A2 * exp(-(double)C2 / TEMP);
  return K1 + K2 * (1.0e+6 * CFACTOR);
}

__device__ __forceinline__ double kpp_fall(double TEMP, double CFACTOR, float A0, float B0,
                                           float C0, float A1, float B1, float C1, float CF) {
  double K0 = (double)A0 * exp(-(double)B0 / TEMP) * pow((TEMP / 300.0), (double)C0);
  double K1 = (double)A1 * exp(-(double)B1 / TEMP) * pow((TEMP / 300.0), (double)C1);
  K0 = K0 * CFACTOR * 1.0e+6;
  K1 = K0 / K1;
  return (K0 / (1.0 + K1)) * pow((double)CF, (1.0 / (1.0 + pow((log10(K1)), 2))));
}

// SUN in [0,1] from the model time: a cosine-shaped day between 4.5 h and
// 19.5 h local time, 0 at night (util/UpdateSun.c:1-20).
__device__ __forceinline__ double kpp_update_sun(double TIME) {
  const double PI = 3.14159265358979;
  const double SunRise = 4.5, SunSet = 19.5;
  double Thour = TIME / 3600.0;
  double Tlocal = Thour - (double)(((int)Thour / 24) * 24);
  if ((Tlocal >= SunRise) && (Tlocal <= SunSet)) {
    double Ttmp = (2.0 * Tlocal - SunRise - SunSet) / (SunSet - SunRise);
    if (Ttmp > 0) Ttmp = Ttmp * Ttmp;
    else Ttmp = -Ttmp * Ttmp;
    return (1.0 + cos(PI * Ttmp)) / 2.0;
  }
  return 0.0;
}
