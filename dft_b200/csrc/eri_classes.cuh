// GENERATED by gen_eri.py -- do not edit by hand.
// Straight-line McMurchie-Davidson bodies for the s/p ERI classes.
#pragma once

template <typename T, int C, int S> struct EriClass;

#define DFTK_N_CLASSES 6

// class 0: (ss|ss), split 0 of 1, ket primitives outside
template <typename T>
struct EriClass<T, 0, 0> {
  static constexpr int LA = 0, LB = 0, LC = 0, LD = 0, L = 0;
  static constexpr int NA = 1, NB = 1, NC = 1, ND = 1;
  static constexpr int NSPLIT = 1, NCD = 1, NI = 1;
  static constexpr int BRA_CLASS = 0, KET_CLASS = 0;
  __device__ static constexpr int cd_c(int m) { constexpr int v[] = {0}; return v[m]; }
  __device__ static constexpr int cd_d(int m) { constexpr int v[] = {0}; return v[m]; }
  // Returns the number of primitive quartets evaluated: both sides'
  // primitive pairs come sorted by descending primitive Schwarz factor q,
  // and the loops stop once q_bra * q_ket < eps (each skipped primitive
  // quartet is bounded by that product, Cauchy-Schwarz per primitive pair).
  __device__ __forceinline__ static int run(
      const T* __restrict__ bra, const float* __restrict__ bra_q, long long bra_stride, int bra_kmax,
      int bra_row, int bra_n,
      const T* __restrict__ ket, const float* __restrict__ ket_q, long long ket_stride, int ket_kmax,
      int ket_row, int ket_n, float eps, T (&I)[NI]) {
    #pragma unroll
    for (int q = 0; q < NI; ++q) I[q] = T(0);
    int evaluated = 0;
    const int bra_st = (int)bra_stride, ket_st = (int)ket_stride;
    const int bra_fs = bra_kmax * bra_st, ket_fs = ket_kmax * ket_st;
    const T* __restrict__ bra_p = bra + bra_row;
    const T* __restrict__ ket_p = ket + ket_row;
    const float* __restrict__ bra_qp = bra_q + bra_row;
    const float* __restrict__ ket_qp = ket_q + ket_row;
    const float bq0 = bra_qp[0];
    #pragma unroll 1
    for (int j = 0; j < ket_n; ++j) {
      const float qo = __ldg(ket_qp + j * ket_st);
      if (qo * bq0 < eps) break;
      const T* __restrict__ krec = ket_p + j * ket_st;
      const T kPx = __ldg(krec + 0);
      const T kPy = __ldg(krec + ket_fs);
      const T kPz = __ldg(krec + 2 * ket_fs);
      const T kp = __ldg(krec + 3 * ket_fs);
      const T kK = __ldg(krec + 4 * ket_fs);
      T V0_000 = T(0);
      float bnq = __ldg(bra_qp);
      T bnPx = __ldg(bra_p + 0), bnPy = __ldg(bra_p + bra_fs), bnPz = __ldg(bra_p + 2 * bra_fs), bnp = __ldg(bra_p + 3 * bra_fs), bnK = __ldg(bra_p + 4 * bra_fs);
      #pragma unroll 1
      for (int i = 0; i < bra_n; ++i) {
        const float bcq = bnq;
        const T bPx = bnPx, bPy = bnPy, bPz = bnPz, bp = bnp, bK = bnK;
        if (qo * bcq < eps) break;
        const int in = i + 1 < bra_n ? i + 1 : i;
        bnq = __ldg(bra_qp + in * bra_st);
        const T* __restrict__ bnrec = bra_p + in * bra_st;
        bnPx = __ldg(bnrec + 0);
        bnPy = __ldg(bnrec + bra_fs);
        bnPz = __ldg(bnrec + 2 * bra_fs);
        bnp = __ldg(bnrec + 3 * bra_fs);
        bnK = __ldg(bnrec + 4 * bra_fs);
        ++evaluated;
        const T s = bp + kp;
        const T rs = Math<T>::rsqrt(s);
        const T rho = bp * kp * (rs * rs);
        const T X = bPx - kPx, Y = bPy - kPy, Z = bPz - kPz;
        const T pre = bK * kK * rs;
        T F[1];
        Boys<T, 0>::eval(rho * (X * X + Y * Y + Z * Z), F);
        T cpow = pre;
        const T R000_0 = cpow * F[0];
        V0_000 += R000_0;
      }
      I[0] += V0_000;
    }
    return evaluated;
  }
};

// class 1: (ps|ss), split 0 of 1, bra primitives outside
template <typename T>
struct EriClass<T, 1, 0> {
  static constexpr int LA = 1, LB = 0, LC = 0, LD = 0, L = 1;
  static constexpr int NA = 3, NB = 1, NC = 1, ND = 1;
  static constexpr int NSPLIT = 1, NCD = 1, NI = 3;
  static constexpr int BRA_CLASS = 1, KET_CLASS = 0;
  __device__ static constexpr int cd_c(int m) { constexpr int v[] = {0}; return v[m]; }
  __device__ static constexpr int cd_d(int m) { constexpr int v[] = {0}; return v[m]; }
  // Returns the number of primitive quartets evaluated: both sides'
  // primitive pairs come sorted by descending primitive Schwarz factor q,
  // and the loops stop once q_bra * q_ket < eps (each skipped primitive
  // quartet is bounded by that product, Cauchy-Schwarz per primitive pair).
  __device__ __forceinline__ static int run(
      const T* __restrict__ bra, const float* __restrict__ bra_q, long long bra_stride, int bra_kmax,
      int bra_row, int bra_n,
      const T* __restrict__ ket, const float* __restrict__ ket_q, long long ket_stride, int ket_kmax,
      int ket_row, int ket_n, float eps, T (&I)[NI]) {
    #pragma unroll
    for (int q = 0; q < NI; ++q) I[q] = T(0);
    int evaluated = 0;
    const int bra_st = (int)bra_stride, ket_st = (int)ket_stride;
    const int bra_fs = bra_kmax * bra_st, ket_fs = ket_kmax * ket_st;
    const T* __restrict__ bra_p = bra + bra_row;
    const T* __restrict__ ket_p = ket + ket_row;
    const float* __restrict__ bra_qp = bra_q + bra_row;
    const float* __restrict__ ket_qp = ket_q + ket_row;
    const float kq0 = ket_qp[0];
    #pragma unroll 1
    for (int i = 0; i < bra_n; ++i) {
      const float qo = __ldg(bra_qp + i * bra_st);
      if (qo * kq0 < eps) break;
      const T* __restrict__ brec = bra_p + i * bra_st;
      const T bPx = __ldg(brec + 0);
      const T bPy = __ldg(brec + bra_fs);
      const T bPz = __ldg(brec + 2 * bra_fs);
      const T bp = __ldg(brec + 3 * bra_fs);
      const T bK = __ldg(brec + 4 * bra_fs);
      const T bh = __ldg(brec + 5 * bra_fs);
      const T bAx = __ldg(brec + 6 * bra_fs);
      const T bAy = __ldg(brec + 7 * bra_fs);
      const T bAz = __ldg(brec + 8 * bra_fs);
      T W0_000 = T(0), W0_001 = T(0), W0_010 = T(0), W0_100 = T(0);
      if constexpr (sizeof(T) == 4) {
        float knq = __ldg(ket_qp);
        T knPx = __ldg(ket_p + 0), knPy = __ldg(ket_p + ket_fs), knPz = __ldg(ket_p + 2 * ket_fs), knp = __ldg(ket_p + 3 * ket_fs), knK = __ldg(ket_p + 4 * ket_fs);
        #pragma unroll 1
        for (int j = 0; j < ket_n; ++j) {
          const float kcq = knq;
          const T kPx = knPx, kPy = knPy, kPz = knPz, kp = knp, kK = knK;
          if (qo * kcq < eps) break;
          const int jn = j + 1 < ket_n ? j + 1 : j;
          knq = __ldg(ket_qp + jn * ket_st);
          const T* __restrict__ knrec = ket_p + jn * ket_st;
          knPx = __ldg(knrec + 0);
          knPy = __ldg(knrec + ket_fs);
          knPz = __ldg(knrec + 2 * ket_fs);
          knp = __ldg(knrec + 3 * ket_fs);
          knK = __ldg(knrec + 4 * ket_fs);
          ++evaluated;
          const T s = bp + kp;
          const T rs = Math<T>::rsqrt(s);
          const T rho = bp * kp * (rs * rs);
          const T X = bPx - kPx, Y = bPy - kPy, Z = bPz - kPz;
          const T pre = bK * kK * rs;
          const T m2rho = T(-2) * rho;
          T F[2];
          Boys<T, 1>::eval(rho * (X * X + Y * Y + Z * Z), F);
          T cpow = pre;
          const T R000_0 = cpow * F[0];
          cpow *= m2rho;
          const T R000_1 = cpow * F[1];
          const T R001_0 = Z * R000_1;
          const T R010_0 = Y * R000_1;
          const T R100_0 = X * R000_1;
          W0_000 += R000_0;
          W0_001 += R001_0;
          W0_010 += R010_0;
          W0_100 += R100_0;
        }
      } else {
        #pragma unroll 1
        for (int j = 0; j < ket_n; ++j) {
          if (qo * __ldg(ket_qp + j * ket_st) < eps) break;
          const T* __restrict__ krec = ket_p + j * ket_st;
          const T kPx = __ldg(krec + 0);
          const T kPy = __ldg(krec + ket_fs);
          const T kPz = __ldg(krec + 2 * ket_fs);
          const T kp = __ldg(krec + 3 * ket_fs);
          const T kK = __ldg(krec + 4 * ket_fs);
          ++evaluated;
          const T s = bp + kp;
          const T rs = Math<T>::rsqrt(s);
          const T rho = bp * kp * (rs * rs);
          const T X = bPx - kPx, Y = bPy - kPy, Z = bPz - kPz;
          const T pre = bK * kK * rs;
          const T m2rho = T(-2) * rho;
          T F[2];
          Boys<T, 1>::eval(rho * (X * X + Y * Y + Z * Z), F);
          T cpow = pre;
          const T R000_0 = cpow * F[0];
          cpow *= m2rho;
          const T R000_1 = cpow * F[1];
          const T R001_0 = Z * R000_1;
          const T R010_0 = Y * R000_1;
          const T R100_0 = X * R000_1;
          W0_000 += R000_0;
          W0_001 += R001_0;
          W0_010 += R010_0;
          W0_100 += R100_0;
        }
      }
      I[0] = fma(bAx, W0_000, I[0]);
      I[0] = fma(bh, W0_100, I[0]);
      I[1] = fma(bAy, W0_000, I[1]);
      I[1] = fma(bh, W0_010, I[1]);
      I[2] = fma(bAz, W0_000, I[2]);
      I[2] = fma(bh, W0_001, I[2]);
    }
    return evaluated;
  }
};

// class 2: (ps|ps), split 0 of 1, ket primitives outside
template <typename T>
struct EriClass<T, 2, 0> {
  static constexpr int LA = 1, LB = 0, LC = 1, LD = 0, L = 2;
  static constexpr int NA = 3, NB = 1, NC = 3, ND = 1;
  static constexpr int NSPLIT = 1, NCD = 3, NI = 9;
  static constexpr int BRA_CLASS = 1, KET_CLASS = 1;
  __device__ static constexpr int cd_c(int m) { constexpr int v[] = {0, 1, 2}; return v[m]; }
  __device__ static constexpr int cd_d(int m) { constexpr int v[] = {0, 0, 0}; return v[m]; }
  // Returns the number of primitive quartets evaluated: both sides'
  // primitive pairs come sorted by descending primitive Schwarz factor q,
  // and the loops stop once q_bra * q_ket < eps (each skipped primitive
  // quartet is bounded by that product, Cauchy-Schwarz per primitive pair).
  __device__ __forceinline__ static int run(
      const T* __restrict__ bra, const float* __restrict__ bra_q, long long bra_stride, int bra_kmax,
      int bra_row, int bra_n,
      const T* __restrict__ ket, const float* __restrict__ ket_q, long long ket_stride, int ket_kmax,
      int ket_row, int ket_n, float eps, T (&I)[NI]) {
    #pragma unroll
    for (int q = 0; q < NI; ++q) I[q] = T(0);
    int evaluated = 0;
    const int bra_st = (int)bra_stride, ket_st = (int)ket_stride;
    const int bra_fs = bra_kmax * bra_st, ket_fs = ket_kmax * ket_st;
    const T* __restrict__ bra_p = bra + bra_row;
    const T* __restrict__ ket_p = ket + ket_row;
    const float* __restrict__ bra_qp = bra_q + bra_row;
    const float* __restrict__ ket_qp = ket_q + ket_row;
    const float bq0 = bra_qp[0];
    #pragma unroll 1
    for (int j = 0; j < ket_n; ++j) {
      const float qo = __ldg(ket_qp + j * ket_st);
      if (qo * bq0 < eps) break;
      const T* __restrict__ krec = ket_p + j * ket_st;
      const T kPx = __ldg(krec + 0);
      const T kPy = __ldg(krec + ket_fs);
      const T kPz = __ldg(krec + 2 * ket_fs);
      const T kp = __ldg(krec + 3 * ket_fs);
      const T kK = __ldg(krec + 4 * ket_fs);
      T V0_000 = T(0), V0_001 = T(0), V0_010 = T(0), V0_100 = T(0);
      T V1_000 = T(0), V1_001 = T(0), V1_010 = T(0), V1_100 = T(0);
      T V2_000 = T(0), V2_001 = T(0), V2_010 = T(0), V2_100 = T(0);
      #pragma unroll 1
      for (int i = 0; i < bra_n; ++i) {
        if (qo * __ldg(bra_qp + i * bra_st) < eps) break;
        const T* __restrict__ brec = bra_p + i * bra_st;
        const T bPx = __ldg(brec + 0);
        const T bPy = __ldg(brec + bra_fs);
        const T bPz = __ldg(brec + 2 * bra_fs);
        const T bp = __ldg(brec + 3 * bra_fs);
        const T bK = __ldg(brec + 4 * bra_fs);
        const T bh = __ldg(brec + 5 * bra_fs);
        const T bAx = __ldg(brec + 6 * bra_fs);
        const T bAy = __ldg(brec + 7 * bra_fs);
        const T bAz = __ldg(brec + 8 * bra_fs);
        ++evaluated;
        const T s = bp + kp;
        const T rs = Math<T>::rsqrt(s);
        const T rho = bp * kp * (rs * rs);
        const T X = bPx - kPx, Y = bPy - kPy, Z = bPz - kPz;
        const T pre = bK * kK * rs;
        const T m2rho = T(-2) * rho;
        T F[3];
        Boys<T, 2>::eval(rho * (X * X + Y * Y + Z * Z), F);
        T cpow = pre;
        const T R000_0 = cpow * F[0];
        cpow *= m2rho;
        const T R000_1 = cpow * F[1];
        cpow *= m2rho;
        const T R000_2 = cpow * F[2];
        const T R001_1 = Z * R000_2;
        const T R010_1 = Y * R000_2;
        const T R100_1 = X * R000_2;
        const T R001_0 = Z * R000_1;
        const T R010_0 = Y * R000_1;
        const T R100_0 = X * R000_1;
        const T R002_0 = Z * R001_1 + T(1) * R000_1;
        const T R011_0 = Y * R001_1;
        const T R020_0 = Y * R010_1 + T(1) * R000_1;
        const T R101_0 = X * R001_1;
        const T R110_0 = X * R010_1;
        const T R200_0 = X * R100_1 + T(1) * R000_1;
        const T bc0_000 = bAx;
        V0_000 = fma(bc0_000, R000_0, V0_000);
        V0_001 = fma(bc0_000, R001_0, V0_001);
        V0_010 = fma(bc0_000, R010_0, V0_010);
        V0_100 = fma(bc0_000, R100_0, V0_100);
        const T bc0_100 = bh;
        V0_000 = fma(bc0_100, R100_0, V0_000);
        V0_001 = fma(bc0_100, R101_0, V0_001);
        V0_010 = fma(bc0_100, R110_0, V0_010);
        V0_100 = fma(bc0_100, R200_0, V0_100);
        const T bc1_000 = bAy;
        V1_000 = fma(bc1_000, R000_0, V1_000);
        V1_001 = fma(bc1_000, R001_0, V1_001);
        V1_010 = fma(bc1_000, R010_0, V1_010);
        V1_100 = fma(bc1_000, R100_0, V1_100);
        const T bc1_010 = bh;
        V1_000 = fma(bc1_010, R010_0, V1_000);
        V1_001 = fma(bc1_010, R011_0, V1_001);
        V1_010 = fma(bc1_010, R020_0, V1_010);
        V1_100 = fma(bc1_010, R110_0, V1_100);
        const T bc2_000 = bAz;
        V2_000 = fma(bc2_000, R000_0, V2_000);
        V2_001 = fma(bc2_000, R001_0, V2_001);
        V2_010 = fma(bc2_000, R010_0, V2_010);
        V2_100 = fma(bc2_000, R100_0, V2_100);
        const T bc2_001 = bh;
        V2_000 = fma(bc2_001, R001_0, V2_000);
        V2_001 = fma(bc2_001, R002_0, V2_001);
        V2_010 = fma(bc2_001, R011_0, V2_010);
        V2_100 = fma(bc2_001, R101_0, V2_100);
      }
      const T kh = __ldg(krec + 5 * ket_fs);
      const T kAx = __ldg(krec + 6 * ket_fs);
      const T kAy = __ldg(krec + 7 * ket_fs);
      const T kAz = __ldg(krec + 8 * ket_fs);
      I[0] = fma(kAx, V0_000, I[0]);
      I[0] = fma(-kh, V0_100, I[0]);
      I[3] = fma(kAx, V1_000, I[3]);
      I[3] = fma(-kh, V1_100, I[3]);
      I[6] = fma(kAx, V2_000, I[6]);
      I[6] = fma(-kh, V2_100, I[6]);
      I[1] = fma(kAy, V0_000, I[1]);
      I[1] = fma(-kh, V0_010, I[1]);
      I[4] = fma(kAy, V1_000, I[4]);
      I[4] = fma(-kh, V1_010, I[4]);
      I[7] = fma(kAy, V2_000, I[7]);
      I[7] = fma(-kh, V2_010, I[7]);
      I[2] = fma(kAz, V0_000, I[2]);
      I[2] = fma(-kh, V0_001, I[2]);
      I[5] = fma(kAz, V1_000, I[5]);
      I[5] = fma(-kh, V1_001, I[5]);
      I[8] = fma(kAz, V2_000, I[8]);
      I[8] = fma(-kh, V2_001, I[8]);
    }
    return evaluated;
  }
};

// class 3: (pp|ss), split 0 of 1, bra primitives outside
template <typename T>
struct EriClass<T, 3, 0> {
  static constexpr int LA = 1, LB = 1, LC = 0, LD = 0, L = 2;
  static constexpr int NA = 3, NB = 3, NC = 1, ND = 1;
  static constexpr int NSPLIT = 1, NCD = 1, NI = 9;
  static constexpr int BRA_CLASS = 2, KET_CLASS = 0;
  __device__ static constexpr int cd_c(int m) { constexpr int v[] = {0}; return v[m]; }
  __device__ static constexpr int cd_d(int m) { constexpr int v[] = {0}; return v[m]; }
  // Returns the number of primitive quartets evaluated: both sides'
  // primitive pairs come sorted by descending primitive Schwarz factor q,
  // and the loops stop once q_bra * q_ket < eps (each skipped primitive
  // quartet is bounded by that product, Cauchy-Schwarz per primitive pair).
  __device__ __forceinline__ static int run(
      const T* __restrict__ bra, const float* __restrict__ bra_q, long long bra_stride, int bra_kmax,
      int bra_row, int bra_n,
      const T* __restrict__ ket, const float* __restrict__ ket_q, long long ket_stride, int ket_kmax,
      int ket_row, int ket_n, float eps, T (&I)[NI]) {
    #pragma unroll
    for (int q = 0; q < NI; ++q) I[q] = T(0);
    int evaluated = 0;
    const int bra_st = (int)bra_stride, ket_st = (int)ket_stride;
    const int bra_fs = bra_kmax * bra_st, ket_fs = ket_kmax * ket_st;
    const T* __restrict__ bra_p = bra + bra_row;
    const T* __restrict__ ket_p = ket + ket_row;
    const float* __restrict__ bra_qp = bra_q + bra_row;
    const float* __restrict__ ket_qp = ket_q + ket_row;
    const float kq0 = ket_qp[0];
    #pragma unroll 1
    for (int i = 0; i < bra_n; ++i) {
      const float qo = __ldg(bra_qp + i * bra_st);
      if (qo * kq0 < eps) break;
      const T* __restrict__ brec = bra_p + i * bra_st;
      const T bPx = __ldg(brec + 0);
      const T bPy = __ldg(brec + bra_fs);
      const T bPz = __ldg(brec + 2 * bra_fs);
      const T bp = __ldg(brec + 3 * bra_fs);
      const T bK = __ldg(brec + 4 * bra_fs);
      T W0_000 = T(0), W0_001 = T(0), W0_002 = T(0), W0_010 = T(0), W0_011 = T(0), W0_020 = T(0), W0_100 = T(0), W0_101 = T(0), W0_110 = T(0), W0_200 = T(0);
      float knq = __ldg(ket_qp);
      T knPx = __ldg(ket_p + 0), knPy = __ldg(ket_p + ket_fs), knPz = __ldg(ket_p + 2 * ket_fs), knp = __ldg(ket_p + 3 * ket_fs), knK = __ldg(ket_p + 4 * ket_fs);
      #pragma unroll 1
      for (int j = 0; j < ket_n; ++j) {
        const float kcq = knq;
        const T kPx = knPx, kPy = knPy, kPz = knPz, kp = knp, kK = knK;
        if (qo * kcq < eps) break;
        const int jn = j + 1 < ket_n ? j + 1 : j;
        knq = __ldg(ket_qp + jn * ket_st);
        const T* __restrict__ knrec = ket_p + jn * ket_st;
        knPx = __ldg(knrec + 0);
        knPy = __ldg(knrec + ket_fs);
        knPz = __ldg(knrec + 2 * ket_fs);
        knp = __ldg(knrec + 3 * ket_fs);
        knK = __ldg(knrec + 4 * ket_fs);
        ++evaluated;
        const T s = bp + kp;
        const T rs = Math<T>::rsqrt(s);
        const T rho = bp * kp * (rs * rs);
        const T X = bPx - kPx, Y = bPy - kPy, Z = bPz - kPz;
        const T pre = bK * kK * rs;
        const T m2rho = T(-2) * rho;
        T F[3];
        Boys<T, 2>::eval(rho * (X * X + Y * Y + Z * Z), F);
        T cpow = pre;
        const T R000_0 = cpow * F[0];
        cpow *= m2rho;
        const T R000_1 = cpow * F[1];
        cpow *= m2rho;
        const T R000_2 = cpow * F[2];
        const T R001_1 = Z * R000_2;
        const T R010_1 = Y * R000_2;
        const T R100_1 = X * R000_2;
        const T R001_0 = Z * R000_1;
        const T R010_0 = Y * R000_1;
        const T R100_0 = X * R000_1;
        const T R002_0 = Z * R001_1 + T(1) * R000_1;
        const T R011_0 = Y * R001_1;
        const T R020_0 = Y * R010_1 + T(1) * R000_1;
        const T R101_0 = X * R001_1;
        const T R110_0 = X * R010_1;
        const T R200_0 = X * R100_1 + T(1) * R000_1;
        W0_000 += R000_0;
        W0_001 += R001_0;
        W0_002 += R002_0;
        W0_010 += R010_0;
        W0_011 += R011_0;
        W0_020 += R020_0;
        W0_100 += R100_0;
        W0_101 += R101_0;
        W0_110 += R110_0;
        W0_200 += R200_0;
      }
      const T bh = __ldg(brec + 5 * bra_fs);
      const T bAx = __ldg(brec + 6 * bra_fs);
      const T bAy = __ldg(brec + 7 * bra_fs);
      const T bAz = __ldg(brec + 8 * bra_fs);
      const T bBx = __ldg(brec + 9 * bra_fs);
      const T bBy = __ldg(brec + 10 * bra_fs);
      const T bBz = __ldg(brec + 11 * bra_fs);
      const T bEx0 = bAx * bBx + bh;
      const T bEx1 = bh * (bAx + bBx);
      const T bEy0 = bAy * bBy + bh;
      const T bEy1 = bh * (bAy + bBy);
      const T bEz0 = bAz * bBz + bh;
      const T bEz1 = bh * (bAz + bBz);
      const T bh2 = bh * bh;
      I[0] = fma(bEx0, W0_000, I[0]);
      I[0] = fma(bEx1, W0_100, I[0]);
      I[0] = fma(bh2, W0_200, I[0]);
      I[1] = fma(bAx * bBy, W0_000, I[1]);
      I[1] = fma(bAx * bh, W0_010, I[1]);
      I[1] = fma(bh * bBy, W0_100, I[1]);
      I[1] = fma(bh * bh, W0_110, I[1]);
      I[2] = fma(bAx * bBz, W0_000, I[2]);
      I[2] = fma(bAx * bh, W0_001, I[2]);
      I[2] = fma(bh * bBz, W0_100, I[2]);
      I[2] = fma(bh * bh, W0_101, I[2]);
      I[3] = fma(bBx * bAy, W0_000, I[3]);
      I[3] = fma(bBx * bh, W0_010, I[3]);
      I[3] = fma(bh * bAy, W0_100, I[3]);
      I[3] = fma(bh * bh, W0_110, I[3]);
      I[4] = fma(bEy0, W0_000, I[4]);
      I[4] = fma(bEy1, W0_010, I[4]);
      I[4] = fma(bh2, W0_020, I[4]);
      I[5] = fma(bAy * bBz, W0_000, I[5]);
      I[5] = fma(bAy * bh, W0_001, I[5]);
      I[5] = fma(bh * bBz, W0_010, I[5]);
      I[5] = fma(bh * bh, W0_011, I[5]);
      I[6] = fma(bBx * bAz, W0_000, I[6]);
      I[6] = fma(bBx * bh, W0_001, I[6]);
      I[6] = fma(bh * bAz, W0_100, I[6]);
      I[6] = fma(bh * bh, W0_101, I[6]);
      I[7] = fma(bBy * bAz, W0_000, I[7]);
      I[7] = fma(bBy * bh, W0_001, I[7]);
      I[7] = fma(bh * bAz, W0_010, I[7]);
      I[7] = fma(bh * bh, W0_011, I[7]);
      I[8] = fma(bEz0, W0_000, I[8]);
      I[8] = fma(bEz1, W0_001, I[8]);
      I[8] = fma(bh2, W0_002, I[8]);
    }
    return evaluated;
  }
};

// class 4: (pp|ps), split 0 of 1, bra primitives outside
template <typename T>
struct EriClass<T, 4, 0> {
  static constexpr int LA = 1, LB = 1, LC = 1, LD = 0, L = 3;
  static constexpr int NA = 3, NB = 3, NC = 3, ND = 1;
  static constexpr int NSPLIT = 1, NCD = 3, NI = 27;
  static constexpr int BRA_CLASS = 2, KET_CLASS = 1;
  __device__ static constexpr int cd_c(int m) { constexpr int v[] = {0, 1, 2}; return v[m]; }
  __device__ static constexpr int cd_d(int m) { constexpr int v[] = {0, 0, 0}; return v[m]; }
  // Returns the number of primitive quartets evaluated: both sides'
  // primitive pairs come sorted by descending primitive Schwarz factor q,
  // and the loops stop once q_bra * q_ket < eps (each skipped primitive
  // quartet is bounded by that product, Cauchy-Schwarz per primitive pair).
  __device__ __forceinline__ static int run(
      const T* __restrict__ bra, const float* __restrict__ bra_q, long long bra_stride, int bra_kmax,
      int bra_row, int bra_n,
      const T* __restrict__ ket, const float* __restrict__ ket_q, long long ket_stride, int ket_kmax,
      int ket_row, int ket_n, float eps, T (&I)[NI]) {
    #pragma unroll
    for (int q = 0; q < NI; ++q) I[q] = T(0);
    int evaluated = 0;
    const int bra_st = (int)bra_stride, ket_st = (int)ket_stride;
    const int bra_fs = bra_kmax * bra_st, ket_fs = ket_kmax * ket_st;
    const T* __restrict__ bra_p = bra + bra_row;
    const T* __restrict__ ket_p = ket + ket_row;
    const float* __restrict__ bra_qp = bra_q + bra_row;
    const float* __restrict__ ket_qp = ket_q + ket_row;
    const float kq0 = ket_qp[0];
    #pragma unroll 1
    for (int i = 0; i < bra_n; ++i) {
      const float qo = __ldg(bra_qp + i * bra_st);
      if (qo * kq0 < eps) break;
      const T* __restrict__ brec = bra_p + i * bra_st;
      const T bPx = __ldg(brec + 0);
      const T bPy = __ldg(brec + bra_fs);
      const T bPz = __ldg(brec + 2 * bra_fs);
      const T bp = __ldg(brec + 3 * bra_fs);
      const T bK = __ldg(brec + 4 * bra_fs);
      T W0_000 = T(0), W0_001 = T(0), W0_002 = T(0), W0_010 = T(0), W0_011 = T(0), W0_020 = T(0), W0_100 = T(0), W0_101 = T(0), W0_110 = T(0), W0_200 = T(0);
      T W1_000 = T(0), W1_001 = T(0), W1_002 = T(0), W1_010 = T(0), W1_011 = T(0), W1_020 = T(0), W1_100 = T(0), W1_101 = T(0), W1_110 = T(0), W1_200 = T(0);
      T W2_000 = T(0), W2_001 = T(0), W2_002 = T(0), W2_010 = T(0), W2_011 = T(0), W2_020 = T(0), W2_100 = T(0), W2_101 = T(0), W2_110 = T(0), W2_200 = T(0);
      #pragma unroll 1
      for (int j = 0; j < ket_n; ++j) {
        if (qo * __ldg(ket_qp + j * ket_st) < eps) break;
        const T* __restrict__ krec = ket_p + j * ket_st;
        const T kPx = __ldg(krec + 0);
        const T kPy = __ldg(krec + ket_fs);
        const T kPz = __ldg(krec + 2 * ket_fs);
        const T kp = __ldg(krec + 3 * ket_fs);
        const T kK = __ldg(krec + 4 * ket_fs);
        const T kh = __ldg(krec + 5 * ket_fs);
        const T kAx = __ldg(krec + 6 * ket_fs);
        const T kAy = __ldg(krec + 7 * ket_fs);
        const T kAz = __ldg(krec + 8 * ket_fs);
        ++evaluated;
        const T s = bp + kp;
        const T rs = Math<T>::rsqrt(s);
        const T rho = bp * kp * (rs * rs);
        const T X = bPx - kPx, Y = bPy - kPy, Z = bPz - kPz;
        const T pre = bK * kK * rs;
        const T m2rho = T(-2) * rho;
        T F[4];
        Boys<T, 3>::eval(rho * (X * X + Y * Y + Z * Z), F);
        T cpow = pre;
        const T R000_0 = cpow * F[0];
        cpow *= m2rho;
        const T R000_1 = cpow * F[1];
        cpow *= m2rho;
        const T R000_2 = cpow * F[2];
        cpow *= m2rho;
        const T R000_3 = cpow * F[3];
        const T R001_2 = Z * R000_3;
        const T R010_2 = Y * R000_3;
        const T R100_2 = X * R000_3;
        const T R001_1 = Z * R000_2;
        const T R010_1 = Y * R000_2;
        const T R100_1 = X * R000_2;
        const T R001_0 = Z * R000_1;
        const T R010_0 = Y * R000_1;
        const T R100_0 = X * R000_1;
        const T R002_1 = Z * R001_2 + T(1) * R000_2;
        const T R011_1 = Y * R001_2;
        const T R020_1 = Y * R010_2 + T(1) * R000_2;
        const T R101_1 = X * R001_2;
        const T R110_1 = X * R010_2;
        const T R200_1 = X * R100_2 + T(1) * R000_2;
        const T R002_0 = Z * R001_1 + T(1) * R000_1;
        const T R011_0 = Y * R001_1;
        const T R020_0 = Y * R010_1 + T(1) * R000_1;
        const T R101_0 = X * R001_1;
        const T R110_0 = X * R010_1;
        const T R200_0 = X * R100_1 + T(1) * R000_1;
        const T R003_0 = Z * R002_1 + T(2) * R001_1;
        const T R012_0 = Y * R002_1;
        const T R021_0 = Y * R011_1 + T(1) * R001_1;
        const T R030_0 = Y * R020_1 + T(2) * R010_1;
        const T R102_0 = X * R002_1;
        const T R111_0 = X * R011_1;
        const T R120_0 = X * R020_1;
        const T R201_0 = X * R101_1 + T(1) * R001_1;
        const T R210_0 = X * R110_1 + T(1) * R010_1;
        const T R300_0 = X * R200_1 + T(2) * R100_1;
        const T kc0_000 = kAx;
        W0_000 = fma(kc0_000, R000_0, W0_000);
        W0_001 = fma(kc0_000, R001_0, W0_001);
        W0_002 = fma(kc0_000, R002_0, W0_002);
        W0_010 = fma(kc0_000, R010_0, W0_010);
        W0_011 = fma(kc0_000, R011_0, W0_011);
        W0_020 = fma(kc0_000, R020_0, W0_020);
        W0_100 = fma(kc0_000, R100_0, W0_100);
        W0_101 = fma(kc0_000, R101_0, W0_101);
        W0_110 = fma(kc0_000, R110_0, W0_110);
        W0_200 = fma(kc0_000, R200_0, W0_200);
        const T kc0_100 = -kh;
        W0_000 = fma(kc0_100, R100_0, W0_000);
        W0_001 = fma(kc0_100, R101_0, W0_001);
        W0_002 = fma(kc0_100, R102_0, W0_002);
        W0_010 = fma(kc0_100, R110_0, W0_010);
        W0_011 = fma(kc0_100, R111_0, W0_011);
        W0_020 = fma(kc0_100, R120_0, W0_020);
        W0_100 = fma(kc0_100, R200_0, W0_100);
        W0_101 = fma(kc0_100, R201_0, W0_101);
        W0_110 = fma(kc0_100, R210_0, W0_110);
        W0_200 = fma(kc0_100, R300_0, W0_200);
        const T kc1_000 = kAy;
        W1_000 = fma(kc1_000, R000_0, W1_000);
        W1_001 = fma(kc1_000, R001_0, W1_001);
        W1_002 = fma(kc1_000, R002_0, W1_002);
        W1_010 = fma(kc1_000, R010_0, W1_010);
        W1_011 = fma(kc1_000, R011_0, W1_011);
        W1_020 = fma(kc1_000, R020_0, W1_020);
        W1_100 = fma(kc1_000, R100_0, W1_100);
        W1_101 = fma(kc1_000, R101_0, W1_101);
        W1_110 = fma(kc1_000, R110_0, W1_110);
        W1_200 = fma(kc1_000, R200_0, W1_200);
        const T kc1_010 = -kh;
        W1_000 = fma(kc1_010, R010_0, W1_000);
        W1_001 = fma(kc1_010, R011_0, W1_001);
        W1_002 = fma(kc1_010, R012_0, W1_002);
        W1_010 = fma(kc1_010, R020_0, W1_010);
        W1_011 = fma(kc1_010, R021_0, W1_011);
        W1_020 = fma(kc1_010, R030_0, W1_020);
        W1_100 = fma(kc1_010, R110_0, W1_100);
        W1_101 = fma(kc1_010, R111_0, W1_101);
        W1_110 = fma(kc1_010, R120_0, W1_110);
        W1_200 = fma(kc1_010, R210_0, W1_200);
        const T kc2_000 = kAz;
        W2_000 = fma(kc2_000, R000_0, W2_000);
        W2_001 = fma(kc2_000, R001_0, W2_001);
        W2_002 = fma(kc2_000, R002_0, W2_002);
        W2_010 = fma(kc2_000, R010_0, W2_010);
        W2_011 = fma(kc2_000, R011_0, W2_011);
        W2_020 = fma(kc2_000, R020_0, W2_020);
        W2_100 = fma(kc2_000, R100_0, W2_100);
        W2_101 = fma(kc2_000, R101_0, W2_101);
        W2_110 = fma(kc2_000, R110_0, W2_110);
        W2_200 = fma(kc2_000, R200_0, W2_200);
        const T kc2_001 = -kh;
        W2_000 = fma(kc2_001, R001_0, W2_000);
        W2_001 = fma(kc2_001, R002_0, W2_001);
        W2_002 = fma(kc2_001, R003_0, W2_002);
        W2_010 = fma(kc2_001, R011_0, W2_010);
        W2_011 = fma(kc2_001, R012_0, W2_011);
        W2_020 = fma(kc2_001, R021_0, W2_020);
        W2_100 = fma(kc2_001, R101_0, W2_100);
        W2_101 = fma(kc2_001, R102_0, W2_101);
        W2_110 = fma(kc2_001, R111_0, W2_110);
        W2_200 = fma(kc2_001, R201_0, W2_200);
      }
      const T bh = __ldg(brec + 5 * bra_fs);
      const T bAx = __ldg(brec + 6 * bra_fs);
      const T bAy = __ldg(brec + 7 * bra_fs);
      const T bAz = __ldg(brec + 8 * bra_fs);
      const T bBx = __ldg(brec + 9 * bra_fs);
      const T bBy = __ldg(brec + 10 * bra_fs);
      const T bBz = __ldg(brec + 11 * bra_fs);
      const T bEx0 = bAx * bBx + bh;
      const T bEx1 = bh * (bAx + bBx);
      const T bEy0 = bAy * bBy + bh;
      const T bEy1 = bh * (bAy + bBy);
      const T bEz0 = bAz * bBz + bh;
      const T bEz1 = bh * (bAz + bBz);
      const T bh2 = bh * bh;
      I[0] = fma(bEx0, W0_000, I[0]);
      I[0] = fma(bEx1, W0_100, I[0]);
      I[0] = fma(bh2, W0_200, I[0]);
      I[1] = fma(bEx0, W1_000, I[1]);
      I[1] = fma(bEx1, W1_100, I[1]);
      I[1] = fma(bh2, W1_200, I[1]);
      I[2] = fma(bEx0, W2_000, I[2]);
      I[2] = fma(bEx1, W2_100, I[2]);
      I[2] = fma(bh2, W2_200, I[2]);
      I[3] = fma(bAx * bBy, W0_000, I[3]);
      I[3] = fma(bAx * bh, W0_010, I[3]);
      I[3] = fma(bh * bBy, W0_100, I[3]);
      I[3] = fma(bh * bh, W0_110, I[3]);
      I[4] = fma(bAx * bBy, W1_000, I[4]);
      I[4] = fma(bAx * bh, W1_010, I[4]);
      I[4] = fma(bh * bBy, W1_100, I[4]);
      I[4] = fma(bh * bh, W1_110, I[4]);
      I[5] = fma(bAx * bBy, W2_000, I[5]);
      I[5] = fma(bAx * bh, W2_010, I[5]);
      I[5] = fma(bh * bBy, W2_100, I[5]);
      I[5] = fma(bh * bh, W2_110, I[5]);
      I[6] = fma(bAx * bBz, W0_000, I[6]);
      I[6] = fma(bAx * bh, W0_001, I[6]);
      I[6] = fma(bh * bBz, W0_100, I[6]);
      I[6] = fma(bh * bh, W0_101, I[6]);
      I[7] = fma(bAx * bBz, W1_000, I[7]);
      I[7] = fma(bAx * bh, W1_001, I[7]);
      I[7] = fma(bh * bBz, W1_100, I[7]);
      I[7] = fma(bh * bh, W1_101, I[7]);
      I[8] = fma(bAx * bBz, W2_000, I[8]);
      I[8] = fma(bAx * bh, W2_001, I[8]);
      I[8] = fma(bh * bBz, W2_100, I[8]);
      I[8] = fma(bh * bh, W2_101, I[8]);
      I[9] = fma(bBx * bAy, W0_000, I[9]);
      I[9] = fma(bBx * bh, W0_010, I[9]);
      I[9] = fma(bh * bAy, W0_100, I[9]);
      I[9] = fma(bh * bh, W0_110, I[9]);
      I[10] = fma(bBx * bAy, W1_000, I[10]);
      I[10] = fma(bBx * bh, W1_010, I[10]);
      I[10] = fma(bh * bAy, W1_100, I[10]);
      I[10] = fma(bh * bh, W1_110, I[10]);
      I[11] = fma(bBx * bAy, W2_000, I[11]);
      I[11] = fma(bBx * bh, W2_010, I[11]);
      I[11] = fma(bh * bAy, W2_100, I[11]);
      I[11] = fma(bh * bh, W2_110, I[11]);
      I[12] = fma(bEy0, W0_000, I[12]);
      I[12] = fma(bEy1, W0_010, I[12]);
      I[12] = fma(bh2, W0_020, I[12]);
      I[13] = fma(bEy0, W1_000, I[13]);
      I[13] = fma(bEy1, W1_010, I[13]);
      I[13] = fma(bh2, W1_020, I[13]);
      I[14] = fma(bEy0, W2_000, I[14]);
      I[14] = fma(bEy1, W2_010, I[14]);
      I[14] = fma(bh2, W2_020, I[14]);
      I[15] = fma(bAy * bBz, W0_000, I[15]);
      I[15] = fma(bAy * bh, W0_001, I[15]);
      I[15] = fma(bh * bBz, W0_010, I[15]);
      I[15] = fma(bh * bh, W0_011, I[15]);
      I[16] = fma(bAy * bBz, W1_000, I[16]);
      I[16] = fma(bAy * bh, W1_001, I[16]);
      I[16] = fma(bh * bBz, W1_010, I[16]);
      I[16] = fma(bh * bh, W1_011, I[16]);
      I[17] = fma(bAy * bBz, W2_000, I[17]);
      I[17] = fma(bAy * bh, W2_001, I[17]);
      I[17] = fma(bh * bBz, W2_010, I[17]);
      I[17] = fma(bh * bh, W2_011, I[17]);
      I[18] = fma(bBx * bAz, W0_000, I[18]);
      I[18] = fma(bBx * bh, W0_001, I[18]);
      I[18] = fma(bh * bAz, W0_100, I[18]);
      I[18] = fma(bh * bh, W0_101, I[18]);
      I[19] = fma(bBx * bAz, W1_000, I[19]);
      I[19] = fma(bBx * bh, W1_001, I[19]);
      I[19] = fma(bh * bAz, W1_100, I[19]);
      I[19] = fma(bh * bh, W1_101, I[19]);
      I[20] = fma(bBx * bAz, W2_000, I[20]);
      I[20] = fma(bBx * bh, W2_001, I[20]);
      I[20] = fma(bh * bAz, W2_100, I[20]);
      I[20] = fma(bh * bh, W2_101, I[20]);
      I[21] = fma(bBy * bAz, W0_000, I[21]);
      I[21] = fma(bBy * bh, W0_001, I[21]);
      I[21] = fma(bh * bAz, W0_010, I[21]);
      I[21] = fma(bh * bh, W0_011, I[21]);
      I[22] = fma(bBy * bAz, W1_000, I[22]);
      I[22] = fma(bBy * bh, W1_001, I[22]);
      I[22] = fma(bh * bAz, W1_010, I[22]);
      I[22] = fma(bh * bh, W1_011, I[22]);
      I[23] = fma(bBy * bAz, W2_000, I[23]);
      I[23] = fma(bBy * bh, W2_001, I[23]);
      I[23] = fma(bh * bAz, W2_010, I[23]);
      I[23] = fma(bh * bh, W2_011, I[23]);
      I[24] = fma(bEz0, W0_000, I[24]);
      I[24] = fma(bEz1, W0_001, I[24]);
      I[24] = fma(bh2, W0_002, I[24]);
      I[25] = fma(bEz0, W1_000, I[25]);
      I[25] = fma(bEz1, W1_001, I[25]);
      I[25] = fma(bh2, W1_002, I[25]);
      I[26] = fma(bEz0, W2_000, I[26]);
      I[26] = fma(bEz1, W2_001, I[26]);
      I[26] = fma(bh2, W2_002, I[26]);
    }
    return evaluated;
  }
};

// class 5: (pp|pp), split 0 of 3, bra primitives outside
template <typename T>
struct EriClass<T, 5, 0> {
  static constexpr int LA = 1, LB = 1, LC = 1, LD = 1, L = 4;
  static constexpr int NA = 3, NB = 3, NC = 3, ND = 3;
  static constexpr int NSPLIT = 3, NCD = 3, NI = 27;
  static constexpr int BRA_CLASS = 2, KET_CLASS = 2;
  __device__ static constexpr int cd_c(int m) { constexpr int v[] = {0, 0, 0}; return v[m]; }
  __device__ static constexpr int cd_d(int m) { constexpr int v[] = {0, 1, 2}; return v[m]; }
  // Returns the number of primitive quartets evaluated: both sides'
  // primitive pairs come sorted by descending primitive Schwarz factor q,
  // and the loops stop once q_bra * q_ket < eps (each skipped primitive
  // quartet is bounded by that product, Cauchy-Schwarz per primitive pair).
  __device__ __forceinline__ static int run(
      const T* __restrict__ bra, const float* __restrict__ bra_q, long long bra_stride, int bra_kmax,
      int bra_row, int bra_n,
      const T* __restrict__ ket, const float* __restrict__ ket_q, long long ket_stride, int ket_kmax,
      int ket_row, int ket_n, float eps, T (&I)[NI]) {
    #pragma unroll
    for (int q = 0; q < NI; ++q) I[q] = T(0);
    int evaluated = 0;
    const int bra_st = (int)bra_stride, ket_st = (int)ket_stride;
    const int bra_fs = bra_kmax * bra_st, ket_fs = ket_kmax * ket_st;
    const T* __restrict__ bra_p = bra + bra_row;
    const T* __restrict__ ket_p = ket + ket_row;
    const float* __restrict__ bra_qp = bra_q + bra_row;
    const float* __restrict__ ket_qp = ket_q + ket_row;
    const float kq0 = ket_qp[0];
    #pragma unroll 1
    for (int i = 0; i < bra_n; ++i) {
      const float qo = __ldg(bra_qp + i * bra_st);
      if (qo * kq0 < eps) break;
      const T* __restrict__ brec = bra_p + i * bra_st;
      const T bPx = __ldg(brec + 0);
      const T bPy = __ldg(brec + bra_fs);
      const T bPz = __ldg(brec + 2 * bra_fs);
      const T bp = __ldg(brec + 3 * bra_fs);
      const T bK = __ldg(brec + 4 * bra_fs);
      T W0_000 = T(0), W0_001 = T(0), W0_002 = T(0), W0_010 = T(0), W0_011 = T(0), W0_020 = T(0), W0_100 = T(0), W0_101 = T(0), W0_110 = T(0), W0_200 = T(0);
      T W1_000 = T(0), W1_001 = T(0), W1_002 = T(0), W1_010 = T(0), W1_011 = T(0), W1_020 = T(0), W1_100 = T(0), W1_101 = T(0), W1_110 = T(0), W1_200 = T(0);
      T W2_000 = T(0), W2_001 = T(0), W2_002 = T(0), W2_010 = T(0), W2_011 = T(0), W2_020 = T(0), W2_100 = T(0), W2_101 = T(0), W2_110 = T(0), W2_200 = T(0);
      float knq = __ldg(ket_qp);
      T knPx = __ldg(ket_p + 0), knPy = __ldg(ket_p + ket_fs), knPz = __ldg(ket_p + 2 * ket_fs), knp = __ldg(ket_p + 3 * ket_fs), knK = __ldg(ket_p + 4 * ket_fs), knh = __ldg(ket_p + 5 * ket_fs), knAx = __ldg(ket_p + 6 * ket_fs), knAy = __ldg(ket_p + 7 * ket_fs), knAz = __ldg(ket_p + 8 * ket_fs), knBx = __ldg(ket_p + 9 * ket_fs), knBy = __ldg(ket_p + 10 * ket_fs), knBz = __ldg(ket_p + 11 * ket_fs);
      #pragma unroll 1
      for (int j = 0; j < ket_n; ++j) {
        const float kcq = knq;
        const T kPx = knPx, kPy = knPy, kPz = knPz, kp = knp, kK = knK, kh = knh, kAx = knAx, kAy = knAy, kAz = knAz, kBx = knBx, kBy = knBy, kBz = knBz;
        if (qo * kcq < eps) break;
        const int jn = j + 1 < ket_n ? j + 1 : j;
        knq = __ldg(ket_qp + jn * ket_st);
        const T* __restrict__ knrec = ket_p + jn * ket_st;
        knPx = __ldg(knrec + 0);
        knPy = __ldg(knrec + ket_fs);
        knPz = __ldg(knrec + 2 * ket_fs);
        knp = __ldg(knrec + 3 * ket_fs);
        knK = __ldg(knrec + 4 * ket_fs);
        knh = __ldg(knrec + 5 * ket_fs);
        knAx = __ldg(knrec + 6 * ket_fs);
        knAy = __ldg(knrec + 7 * ket_fs);
        knAz = __ldg(knrec + 8 * ket_fs);
        knBx = __ldg(knrec + 9 * ket_fs);
        knBy = __ldg(knrec + 10 * ket_fs);
        knBz = __ldg(knrec + 11 * ket_fs);
        ++evaluated;
        const T kEx0 = kAx * kBx + kh;
        const T kEx1 = kh * (kAx + kBx);
        const T kEy0 = kAy * kBy + kh;
        const T kEy1 = kh * (kAy + kBy);
        const T kEz0 = kAz * kBz + kh;
        const T kEz1 = kh * (kAz + kBz);
        const T kh2 = kh * kh;
        const T s = bp + kp;
        const T rs = Math<T>::rsqrt(s);
        const T rho = bp * kp * (rs * rs);
        const T X = bPx - kPx, Y = bPy - kPy, Z = bPz - kPz;
        const T pre = bK * kK * rs;
        const T m2rho = T(-2) * rho;
        T F[5];
        Boys<T, 4>::eval(rho * (X * X + Y * Y + Z * Z), F);
        T cpow = pre;
        const T R000_0 = cpow * F[0];
        cpow *= m2rho;
        const T R000_1 = cpow * F[1];
        cpow *= m2rho;
        const T R000_2 = cpow * F[2];
        cpow *= m2rho;
        const T R000_3 = cpow * F[3];
        cpow *= m2rho;
        const T R000_4 = cpow * F[4];
        const T R001_3 = Z * R000_4;
        const T R010_3 = Y * R000_4;
        const T R100_3 = X * R000_4;
        const T R001_2 = Z * R000_3;
        const T R010_2 = Y * R000_3;
        const T R100_2 = X * R000_3;
        const T R001_1 = Z * R000_2;
        const T R010_1 = Y * R000_2;
        const T R100_1 = X * R000_2;
        const T R001_0 = Z * R000_1;
        const T R010_0 = Y * R000_1;
        const T R100_0 = X * R000_1;
        const T R002_2 = Z * R001_3 + T(1) * R000_3;
        const T R011_2 = Y * R001_3;
        const T R020_2 = Y * R010_3 + T(1) * R000_3;
        const T R101_2 = X * R001_3;
        const T R110_2 = X * R010_3;
        const T R200_2 = X * R100_3 + T(1) * R000_3;
        const T R002_1 = Z * R001_2 + T(1) * R000_2;
        const T R011_1 = Y * R001_2;
        const T R020_1 = Y * R010_2 + T(1) * R000_2;
        const T R101_1 = X * R001_2;
        const T R110_1 = X * R010_2;
        const T R200_1 = X * R100_2 + T(1) * R000_2;
        const T R002_0 = Z * R001_1 + T(1) * R000_1;
        const T R011_0 = Y * R001_1;
        const T R020_0 = Y * R010_1 + T(1) * R000_1;
        const T R101_0 = X * R001_1;
        const T R110_0 = X * R010_1;
        const T R200_0 = X * R100_1 + T(1) * R000_1;
        const T R003_1 = Z * R002_2 + T(2) * R001_2;
        const T R012_1 = Y * R002_2;
        const T R021_1 = Y * R011_2 + T(1) * R001_2;
        const T R030_1 = Y * R020_2 + T(2) * R010_2;
        const T R102_1 = X * R002_2;
        const T R111_1 = X * R011_2;
        const T R120_1 = X * R020_2;
        const T R201_1 = X * R101_2 + T(1) * R001_2;
        const T R210_1 = X * R110_2 + T(1) * R010_2;
        const T R300_1 = X * R200_2 + T(2) * R100_2;
        const T R003_0 = Z * R002_1 + T(2) * R001_1;
        const T R012_0 = Y * R002_1;
        const T R021_0 = Y * R011_1 + T(1) * R001_1;
        const T R030_0 = Y * R020_1 + T(2) * R010_1;
        const T R102_0 = X * R002_1;
        const T R111_0 = X * R011_1;
        const T R120_0 = X * R020_1;
        const T R201_0 = X * R101_1 + T(1) * R001_1;
        const T R210_0 = X * R110_1 + T(1) * R010_1;
        const T R300_0 = X * R200_1 + T(2) * R100_1;
        const T R103_0 = X * R003_1;
        const T R112_0 = X * R012_1;
        const T R121_0 = X * R021_1;
        const T R130_0 = X * R030_1;
        const T R202_0 = X * R102_1 + T(1) * R002_1;
        const T R211_0 = X * R111_1 + T(1) * R011_1;
        const T R220_0 = X * R120_1 + T(1) * R020_1;
        const T R301_0 = X * R201_1 + T(2) * R101_1;
        const T R310_0 = X * R210_1 + T(2) * R110_1;
        const T R400_0 = X * R300_1 + T(3) * R200_1;
        const T kc0_000 = kEx0;
        W0_000 = fma(kc0_000, R000_0, W0_000);
        W0_001 = fma(kc0_000, R001_0, W0_001);
        W0_002 = fma(kc0_000, R002_0, W0_002);
        W0_010 = fma(kc0_000, R010_0, W0_010);
        W0_011 = fma(kc0_000, R011_0, W0_011);
        W0_020 = fma(kc0_000, R020_0, W0_020);
        W0_100 = fma(kc0_000, R100_0, W0_100);
        W0_101 = fma(kc0_000, R101_0, W0_101);
        W0_110 = fma(kc0_000, R110_0, W0_110);
        W0_200 = fma(kc0_000, R200_0, W0_200);
        const T kc0_100 = -kEx1;
        W0_000 = fma(kc0_100, R100_0, W0_000);
        W0_001 = fma(kc0_100, R101_0, W0_001);
        W0_002 = fma(kc0_100, R102_0, W0_002);
        W0_010 = fma(kc0_100, R110_0, W0_010);
        W0_011 = fma(kc0_100, R111_0, W0_011);
        W0_020 = fma(kc0_100, R120_0, W0_020);
        W0_100 = fma(kc0_100, R200_0, W0_100);
        W0_101 = fma(kc0_100, R201_0, W0_101);
        W0_110 = fma(kc0_100, R210_0, W0_110);
        W0_200 = fma(kc0_100, R300_0, W0_200);
        const T kc0_200 = kh2;
        W0_000 = fma(kc0_200, R200_0, W0_000);
        W0_001 = fma(kc0_200, R201_0, W0_001);
        W0_002 = fma(kc0_200, R202_0, W0_002);
        W0_010 = fma(kc0_200, R210_0, W0_010);
        W0_011 = fma(kc0_200, R211_0, W0_011);
        W0_020 = fma(kc0_200, R220_0, W0_020);
        W0_100 = fma(kc0_200, R300_0, W0_100);
        W0_101 = fma(kc0_200, R301_0, W0_101);
        W0_110 = fma(kc0_200, R310_0, W0_110);
        W0_200 = fma(kc0_200, R400_0, W0_200);
        const T kc1_000 = kAx * kBy;
        W1_000 = fma(kc1_000, R000_0, W1_000);
        W1_001 = fma(kc1_000, R001_0, W1_001);
        W1_002 = fma(kc1_000, R002_0, W1_002);
        W1_010 = fma(kc1_000, R010_0, W1_010);
        W1_011 = fma(kc1_000, R011_0, W1_011);
        W1_020 = fma(kc1_000, R020_0, W1_020);
        W1_100 = fma(kc1_000, R100_0, W1_100);
        W1_101 = fma(kc1_000, R101_0, W1_101);
        W1_110 = fma(kc1_000, R110_0, W1_110);
        W1_200 = fma(kc1_000, R200_0, W1_200);
        const T kc1_010 = -kAx * kh;
        W1_000 = fma(kc1_010, R010_0, W1_000);
        W1_001 = fma(kc1_010, R011_0, W1_001);
        W1_002 = fma(kc1_010, R012_0, W1_002);
        W1_010 = fma(kc1_010, R020_0, W1_010);
        W1_011 = fma(kc1_010, R021_0, W1_011);
        W1_020 = fma(kc1_010, R030_0, W1_020);
        W1_100 = fma(kc1_010, R110_0, W1_100);
        W1_101 = fma(kc1_010, R111_0, W1_101);
        W1_110 = fma(kc1_010, R120_0, W1_110);
        W1_200 = fma(kc1_010, R210_0, W1_200);
        const T kc1_100 = -kh * kBy;
        W1_000 = fma(kc1_100, R100_0, W1_000);
        W1_001 = fma(kc1_100, R101_0, W1_001);
        W1_002 = fma(kc1_100, R102_0, W1_002);
        W1_010 = fma(kc1_100, R110_0, W1_010);
        W1_011 = fma(kc1_100, R111_0, W1_011);
        W1_020 = fma(kc1_100, R120_0, W1_020);
        W1_100 = fma(kc1_100, R200_0, W1_100);
        W1_101 = fma(kc1_100, R201_0, W1_101);
        W1_110 = fma(kc1_100, R210_0, W1_110);
        W1_200 = fma(kc1_100, R300_0, W1_200);
        const T kc1_110 = kh * kh;
        W1_000 = fma(kc1_110, R110_0, W1_000);
        W1_001 = fma(kc1_110, R111_0, W1_001);
        W1_002 = fma(kc1_110, R112_0, W1_002);
        W1_010 = fma(kc1_110, R120_0, W1_010);
        W1_011 = fma(kc1_110, R121_0, W1_011);
        W1_020 = fma(kc1_110, R130_0, W1_020);
        W1_100 = fma(kc1_110, R210_0, W1_100);
        W1_101 = fma(kc1_110, R211_0, W1_101);
        W1_110 = fma(kc1_110, R220_0, W1_110);
        W1_200 = fma(kc1_110, R310_0, W1_200);
        const T kc2_000 = kAx * kBz;
        W2_000 = fma(kc2_000, R000_0, W2_000);
        W2_001 = fma(kc2_000, R001_0, W2_001);
        W2_002 = fma(kc2_000, R002_0, W2_002);
        W2_010 = fma(kc2_000, R010_0, W2_010);
        W2_011 = fma(kc2_000, R011_0, W2_011);
        W2_020 = fma(kc2_000, R020_0, W2_020);
        W2_100 = fma(kc2_000, R100_0, W2_100);
        W2_101 = fma(kc2_000, R101_0, W2_101);
        W2_110 = fma(kc2_000, R110_0, W2_110);
        W2_200 = fma(kc2_000, R200_0, W2_200);
        const T kc2_001 = -kAx * kh;
        W2_000 = fma(kc2_001, R001_0, W2_000);
        W2_001 = fma(kc2_001, R002_0, W2_001);
        W2_002 = fma(kc2_001, R003_0, W2_002);
        W2_010 = fma(kc2_001, R011_0, W2_010);
        W2_011 = fma(kc2_001, R012_0, W2_011);
        W2_020 = fma(kc2_001, R021_0, W2_020);
        W2_100 = fma(kc2_001, R101_0, W2_100);
        W2_101 = fma(kc2_001, R102_0, W2_101);
        W2_110 = fma(kc2_001, R111_0, W2_110);
        W2_200 = fma(kc2_001, R201_0, W2_200);
        const T kc2_100 = -kh * kBz;
        W2_000 = fma(kc2_100, R100_0, W2_000);
        W2_001 = fma(kc2_100, R101_0, W2_001);
        W2_002 = fma(kc2_100, R102_0, W2_002);
        W2_010 = fma(kc2_100, R110_0, W2_010);
        W2_011 = fma(kc2_100, R111_0, W2_011);
        W2_020 = fma(kc2_100, R120_0, W2_020);
        W2_100 = fma(kc2_100, R200_0, W2_100);
        W2_101 = fma(kc2_100, R201_0, W2_101);
        W2_110 = fma(kc2_100, R210_0, W2_110);
        W2_200 = fma(kc2_100, R300_0, W2_200);
        const T kc2_101 = kh * kh;
        W2_000 = fma(kc2_101, R101_0, W2_000);
        W2_001 = fma(kc2_101, R102_0, W2_001);
        W2_002 = fma(kc2_101, R103_0, W2_002);
        W2_010 = fma(kc2_101, R111_0, W2_010);
        W2_011 = fma(kc2_101, R112_0, W2_011);
        W2_020 = fma(kc2_101, R121_0, W2_020);
        W2_100 = fma(kc2_101, R201_0, W2_100);
        W2_101 = fma(kc2_101, R202_0, W2_101);
        W2_110 = fma(kc2_101, R211_0, W2_110);
        W2_200 = fma(kc2_101, R301_0, W2_200);
      }
      const T bh = __ldg(brec + 5 * bra_fs);
      const T bAx = __ldg(brec + 6 * bra_fs);
      const T bAy = __ldg(brec + 7 * bra_fs);
      const T bAz = __ldg(brec + 8 * bra_fs);
      const T bBx = __ldg(brec + 9 * bra_fs);
      const T bBy = __ldg(brec + 10 * bra_fs);
      const T bBz = __ldg(brec + 11 * bra_fs);
      const T bEx0 = bAx * bBx + bh;
      const T bEx1 = bh * (bAx + bBx);
      const T bEy0 = bAy * bBy + bh;
      const T bEy1 = bh * (bAy + bBy);
      const T bEz0 = bAz * bBz + bh;
      const T bEz1 = bh * (bAz + bBz);
      const T bh2 = bh * bh;
      I[0] = fma(bEx0, W0_000, I[0]);
      I[0] = fma(bEx1, W0_100, I[0]);
      I[0] = fma(bh2, W0_200, I[0]);
      I[1] = fma(bEx0, W1_000, I[1]);
      I[1] = fma(bEx1, W1_100, I[1]);
      I[1] = fma(bh2, W1_200, I[1]);
      I[2] = fma(bEx0, W2_000, I[2]);
      I[2] = fma(bEx1, W2_100, I[2]);
      I[2] = fma(bh2, W2_200, I[2]);
      I[3] = fma(bAx * bBy, W0_000, I[3]);
      I[3] = fma(bAx * bh, W0_010, I[3]);
      I[3] = fma(bh * bBy, W0_100, I[3]);
      I[3] = fma(bh * bh, W0_110, I[3]);
      I[4] = fma(bAx * bBy, W1_000, I[4]);
      I[4] = fma(bAx * bh, W1_010, I[4]);
      I[4] = fma(bh * bBy, W1_100, I[4]);
      I[4] = fma(bh * bh, W1_110, I[4]);
      I[5] = fma(bAx * bBy, W2_000, I[5]);
      I[5] = fma(bAx * bh, W2_010, I[5]);
      I[5] = fma(bh * bBy, W2_100, I[5]);
      I[5] = fma(bh * bh, W2_110, I[5]);
      I[6] = fma(bAx * bBz, W0_000, I[6]);
      I[6] = fma(bAx * bh, W0_001, I[6]);
      I[6] = fma(bh * bBz, W0_100, I[6]);
      I[6] = fma(bh * bh, W0_101, I[6]);
      I[7] = fma(bAx * bBz, W1_000, I[7]);
      I[7] = fma(bAx * bh, W1_001, I[7]);
      I[7] = fma(bh * bBz, W1_100, I[7]);
      I[7] = fma(bh * bh, W1_101, I[7]);
      I[8] = fma(bAx * bBz, W2_000, I[8]);
      I[8] = fma(bAx * bh, W2_001, I[8]);
      I[8] = fma(bh * bBz, W2_100, I[8]);
      I[8] = fma(bh * bh, W2_101, I[8]);
      I[9] = fma(bBx * bAy, W0_000, I[9]);
      I[9] = fma(bBx * bh, W0_010, I[9]);
      I[9] = fma(bh * bAy, W0_100, I[9]);
      I[9] = fma(bh * bh, W0_110, I[9]);
      I[10] = fma(bBx * bAy, W1_000, I[10]);
      I[10] = fma(bBx * bh, W1_010, I[10]);
      I[10] = fma(bh * bAy, W1_100, I[10]);
      I[10] = fma(bh * bh, W1_110, I[10]);
      I[11] = fma(bBx * bAy, W2_000, I[11]);
      I[11] = fma(bBx * bh, W2_010, I[11]);
      I[11] = fma(bh * bAy, W2_100, I[11]);
      I[11] = fma(bh * bh, W2_110, I[11]);
      I[12] = fma(bEy0, W0_000, I[12]);
      I[12] = fma(bEy1, W0_010, I[12]);
      I[12] = fma(bh2, W0_020, I[12]);
      I[13] = fma(bEy0, W1_000, I[13]);
      I[13] = fma(bEy1, W1_010, I[13]);
      I[13] = fma(bh2, W1_020, I[13]);
      I[14] = fma(bEy0, W2_000, I[14]);
      I[14] = fma(bEy1, W2_010, I[14]);
      I[14] = fma(bh2, W2_020, I[14]);
      I[15] = fma(bAy * bBz, W0_000, I[15]);
      I[15] = fma(bAy * bh, W0_001, I[15]);
      I[15] = fma(bh * bBz, W0_010, I[15]);
      I[15] = fma(bh * bh, W0_011, I[15]);
      I[16] = fma(bAy * bBz, W1_000, I[16]);
      I[16] = fma(bAy * bh, W1_001, I[16]);
      I[16] = fma(bh * bBz, W1_010, I[16]);
      I[16] = fma(bh * bh, W1_011, I[16]);
      I[17] = fma(bAy * bBz, W2_000, I[17]);
      I[17] = fma(bAy * bh, W2_001, I[17]);
      I[17] = fma(bh * bBz, W2_010, I[17]);
      I[17] = fma(bh * bh, W2_011, I[17]);
      I[18] = fma(bBx * bAz, W0_000, I[18]);
      I[18] = fma(bBx * bh, W0_001, I[18]);
      I[18] = fma(bh * bAz, W0_100, I[18]);
      I[18] = fma(bh * bh, W0_101, I[18]);
      I[19] = fma(bBx * bAz, W1_000, I[19]);
      I[19] = fma(bBx * bh, W1_001, I[19]);
      I[19] = fma(bh * bAz, W1_100, I[19]);
      I[19] = fma(bh * bh, W1_101, I[19]);
      I[20] = fma(bBx * bAz, W2_000, I[20]);
      I[20] = fma(bBx * bh, W2_001, I[20]);
      I[20] = fma(bh * bAz, W2_100, I[20]);
      I[20] = fma(bh * bh, W2_101, I[20]);
      I[21] = fma(bBy * bAz, W0_000, I[21]);
      I[21] = fma(bBy * bh, W0_001, I[21]);
      I[21] = fma(bh * bAz, W0_010, I[21]);
      I[21] = fma(bh * bh, W0_011, I[21]);
      I[22] = fma(bBy * bAz, W1_000, I[22]);
      I[22] = fma(bBy * bh, W1_001, I[22]);
      I[22] = fma(bh * bAz, W1_010, I[22]);
      I[22] = fma(bh * bh, W1_011, I[22]);
      I[23] = fma(bBy * bAz, W2_000, I[23]);
      I[23] = fma(bBy * bh, W2_001, I[23]);
      I[23] = fma(bh * bAz, W2_010, I[23]);
      I[23] = fma(bh * bh, W2_011, I[23]);
      I[24] = fma(bEz0, W0_000, I[24]);
      I[24] = fma(bEz1, W0_001, I[24]);
      I[24] = fma(bh2, W0_002, I[24]);
      I[25] = fma(bEz0, W1_000, I[25]);
      I[25] = fma(bEz1, W1_001, I[25]);
      I[25] = fma(bh2, W1_002, I[25]);
      I[26] = fma(bEz0, W2_000, I[26]);
      I[26] = fma(bEz1, W2_001, I[26]);
      I[26] = fma(bh2, W2_002, I[26]);
    }
    return evaluated;
  }
};

// class 5: (pp|pp), split 1 of 3, bra primitives outside
template <typename T>
struct EriClass<T, 5, 1> {
  static constexpr int LA = 1, LB = 1, LC = 1, LD = 1, L = 4;
  static constexpr int NA = 3, NB = 3, NC = 3, ND = 3;
  static constexpr int NSPLIT = 3, NCD = 3, NI = 27;
  static constexpr int BRA_CLASS = 2, KET_CLASS = 2;
  __device__ static constexpr int cd_c(int m) { constexpr int v[] = {1, 1, 1}; return v[m]; }
  __device__ static constexpr int cd_d(int m) { constexpr int v[] = {0, 1, 2}; return v[m]; }
  // Returns the number of primitive quartets evaluated: both sides'
  // primitive pairs come sorted by descending primitive Schwarz factor q,
  // and the loops stop once q_bra * q_ket < eps (each skipped primitive
  // quartet is bounded by that product, Cauchy-Schwarz per primitive pair).
  __device__ __forceinline__ static int run(
      const T* __restrict__ bra, const float* __restrict__ bra_q, long long bra_stride, int bra_kmax,
      int bra_row, int bra_n,
      const T* __restrict__ ket, const float* __restrict__ ket_q, long long ket_stride, int ket_kmax,
      int ket_row, int ket_n, float eps, T (&I)[NI]) {
    #pragma unroll
    for (int q = 0; q < NI; ++q) I[q] = T(0);
    int evaluated = 0;
    const int bra_st = (int)bra_stride, ket_st = (int)ket_stride;
    const int bra_fs = bra_kmax * bra_st, ket_fs = ket_kmax * ket_st;
    const T* __restrict__ bra_p = bra + bra_row;
    const T* __restrict__ ket_p = ket + ket_row;
    const float* __restrict__ bra_qp = bra_q + bra_row;
    const float* __restrict__ ket_qp = ket_q + ket_row;
    const float kq0 = ket_qp[0];
    #pragma unroll 1
    for (int i = 0; i < bra_n; ++i) {
      const float qo = __ldg(bra_qp + i * bra_st);
      if (qo * kq0 < eps) break;
      const T* __restrict__ brec = bra_p + i * bra_st;
      const T bPx = __ldg(brec + 0);
      const T bPy = __ldg(brec + bra_fs);
      const T bPz = __ldg(brec + 2 * bra_fs);
      const T bp = __ldg(brec + 3 * bra_fs);
      const T bK = __ldg(brec + 4 * bra_fs);
      T W0_000 = T(0), W0_001 = T(0), W0_002 = T(0), W0_010 = T(0), W0_011 = T(0), W0_020 = T(0), W0_100 = T(0), W0_101 = T(0), W0_110 = T(0), W0_200 = T(0);
      T W1_000 = T(0), W1_001 = T(0), W1_002 = T(0), W1_010 = T(0), W1_011 = T(0), W1_020 = T(0), W1_100 = T(0), W1_101 = T(0), W1_110 = T(0), W1_200 = T(0);
      T W2_000 = T(0), W2_001 = T(0), W2_002 = T(0), W2_010 = T(0), W2_011 = T(0), W2_020 = T(0), W2_100 = T(0), W2_101 = T(0), W2_110 = T(0), W2_200 = T(0);
      float knq = __ldg(ket_qp);
      T knPx = __ldg(ket_p + 0), knPy = __ldg(ket_p + ket_fs), knPz = __ldg(ket_p + 2 * ket_fs), knp = __ldg(ket_p + 3 * ket_fs), knK = __ldg(ket_p + 4 * ket_fs), knh = __ldg(ket_p + 5 * ket_fs), knAx = __ldg(ket_p + 6 * ket_fs), knAy = __ldg(ket_p + 7 * ket_fs), knAz = __ldg(ket_p + 8 * ket_fs), knBx = __ldg(ket_p + 9 * ket_fs), knBy = __ldg(ket_p + 10 * ket_fs), knBz = __ldg(ket_p + 11 * ket_fs);
      #pragma unroll 1
      for (int j = 0; j < ket_n; ++j) {
        const float kcq = knq;
        const T kPx = knPx, kPy = knPy, kPz = knPz, kp = knp, kK = knK, kh = knh, kAx = knAx, kAy = knAy, kAz = knAz, kBx = knBx, kBy = knBy, kBz = knBz;
        if (qo * kcq < eps) break;
        const int jn = j + 1 < ket_n ? j + 1 : j;
        knq = __ldg(ket_qp + jn * ket_st);
        const T* __restrict__ knrec = ket_p + jn * ket_st;
        knPx = __ldg(knrec + 0);
        knPy = __ldg(knrec + ket_fs);
        knPz = __ldg(knrec + 2 * ket_fs);
        knp = __ldg(knrec + 3 * ket_fs);
        knK = __ldg(knrec + 4 * ket_fs);
        knh = __ldg(knrec + 5 * ket_fs);
        knAx = __ldg(knrec + 6 * ket_fs);
        knAy = __ldg(knrec + 7 * ket_fs);
        knAz = __ldg(knrec + 8 * ket_fs);
        knBx = __ldg(knrec + 9 * ket_fs);
        knBy = __ldg(knrec + 10 * ket_fs);
        knBz = __ldg(knrec + 11 * ket_fs);
        ++evaluated;
        const T kEx0 = kAx * kBx + kh;
        const T kEx1 = kh * (kAx + kBx);
        const T kEy0 = kAy * kBy + kh;
        const T kEy1 = kh * (kAy + kBy);
        const T kEz0 = kAz * kBz + kh;
        const T kEz1 = kh * (kAz + kBz);
        const T kh2 = kh * kh;
        const T s = bp + kp;
        const T rs = Math<T>::rsqrt(s);
        const T rho = bp * kp * (rs * rs);
        const T X = bPx - kPx, Y = bPy - kPy, Z = bPz - kPz;
        const T pre = bK * kK * rs;
        const T m2rho = T(-2) * rho;
        T F[5];
        Boys<T, 4>::eval(rho * (X * X + Y * Y + Z * Z), F);
        T cpow = pre;
        const T R000_0 = cpow * F[0];
        cpow *= m2rho;
        const T R000_1 = cpow * F[1];
        cpow *= m2rho;
        const T R000_2 = cpow * F[2];
        cpow *= m2rho;
        const T R000_3 = cpow * F[3];
        cpow *= m2rho;
        const T R000_4 = cpow * F[4];
        const T R001_3 = Z * R000_4;
        const T R010_3 = Y * R000_4;
        const T R001_2 = Z * R000_3;
        const T R010_2 = Y * R000_3;
        const T R100_2 = X * R000_3;
        const T R001_1 = Z * R000_2;
        const T R010_1 = Y * R000_2;
        const T R100_1 = X * R000_2;
        const T R001_0 = Z * R000_1;
        const T R010_0 = Y * R000_1;
        const T R100_0 = X * R000_1;
        const T R002_2 = Z * R001_3 + T(1) * R000_3;
        const T R011_2 = Y * R001_3;
        const T R020_2 = Y * R010_3 + T(1) * R000_3;
        const T R110_2 = X * R010_3;
        const T R002_1 = Z * R001_2 + T(1) * R000_2;
        const T R011_1 = Y * R001_2;
        const T R020_1 = Y * R010_2 + T(1) * R000_2;
        const T R101_1 = X * R001_2;
        const T R110_1 = X * R010_2;
        const T R200_1 = X * R100_2 + T(1) * R000_2;
        const T R002_0 = Z * R001_1 + T(1) * R000_1;
        const T R011_0 = Y * R001_1;
        const T R020_0 = Y * R010_1 + T(1) * R000_1;
        const T R101_0 = X * R001_1;
        const T R110_0 = X * R010_1;
        const T R200_0 = X * R100_1 + T(1) * R000_1;
        const T R003_1 = Z * R002_2 + T(2) * R001_2;
        const T R012_1 = Y * R002_2;
        const T R021_1 = Y * R011_2 + T(1) * R001_2;
        const T R030_1 = Y * R020_2 + T(2) * R010_2;
        const T R111_1 = X * R011_2;
        const T R120_1 = X * R020_2;
        const T R210_1 = X * R110_2 + T(1) * R010_2;
        const T R003_0 = Z * R002_1 + T(2) * R001_1;
        const T R012_0 = Y * R002_1;
        const T R021_0 = Y * R011_1 + T(1) * R001_1;
        const T R030_0 = Y * R020_1 + T(2) * R010_1;
        const T R102_0 = X * R002_1;
        const T R111_0 = X * R011_1;
        const T R120_0 = X * R020_1;
        const T R201_0 = X * R101_1 + T(1) * R001_1;
        const T R210_0 = X * R110_1 + T(1) * R010_1;
        const T R300_0 = X * R200_1 + T(2) * R100_1;
        const T R013_0 = Y * R003_1;
        const T R022_0 = Y * R012_1 + T(1) * R002_1;
        const T R031_0 = Y * R021_1 + T(2) * R011_1;
        const T R040_0 = Y * R030_1 + T(3) * R020_1;
        const T R112_0 = X * R012_1;
        const T R121_0 = X * R021_1;
        const T R130_0 = X * R030_1;
        const T R211_0 = X * R111_1 + T(1) * R011_1;
        const T R220_0 = X * R120_1 + T(1) * R020_1;
        const T R310_0 = X * R210_1 + T(2) * R110_1;
        const T kc0_000 = kBx * kAy;
        W0_000 = fma(kc0_000, R000_0, W0_000);
        W0_001 = fma(kc0_000, R001_0, W0_001);
        W0_002 = fma(kc0_000, R002_0, W0_002);
        W0_010 = fma(kc0_000, R010_0, W0_010);
        W0_011 = fma(kc0_000, R011_0, W0_011);
        W0_020 = fma(kc0_000, R020_0, W0_020);
        W0_100 = fma(kc0_000, R100_0, W0_100);
        W0_101 = fma(kc0_000, R101_0, W0_101);
        W0_110 = fma(kc0_000, R110_0, W0_110);
        W0_200 = fma(kc0_000, R200_0, W0_200);
        const T kc0_010 = -kBx * kh;
        W0_000 = fma(kc0_010, R010_0, W0_000);
        W0_001 = fma(kc0_010, R011_0, W0_001);
        W0_002 = fma(kc0_010, R012_0, W0_002);
        W0_010 = fma(kc0_010, R020_0, W0_010);
        W0_011 = fma(kc0_010, R021_0, W0_011);
        W0_020 = fma(kc0_010, R030_0, W0_020);
        W0_100 = fma(kc0_010, R110_0, W0_100);
        W0_101 = fma(kc0_010, R111_0, W0_101);
        W0_110 = fma(kc0_010, R120_0, W0_110);
        W0_200 = fma(kc0_010, R210_0, W0_200);
        const T kc0_100 = -kh * kAy;
        W0_000 = fma(kc0_100, R100_0, W0_000);
        W0_001 = fma(kc0_100, R101_0, W0_001);
        W0_002 = fma(kc0_100, R102_0, W0_002);
        W0_010 = fma(kc0_100, R110_0, W0_010);
        W0_011 = fma(kc0_100, R111_0, W0_011);
        W0_020 = fma(kc0_100, R120_0, W0_020);
        W0_100 = fma(kc0_100, R200_0, W0_100);
        W0_101 = fma(kc0_100, R201_0, W0_101);
        W0_110 = fma(kc0_100, R210_0, W0_110);
        W0_200 = fma(kc0_100, R300_0, W0_200);
        const T kc0_110 = kh * kh;
        W0_000 = fma(kc0_110, R110_0, W0_000);
        W0_001 = fma(kc0_110, R111_0, W0_001);
        W0_002 = fma(kc0_110, R112_0, W0_002);
        W0_010 = fma(kc0_110, R120_0, W0_010);
        W0_011 = fma(kc0_110, R121_0, W0_011);
        W0_020 = fma(kc0_110, R130_0, W0_020);
        W0_100 = fma(kc0_110, R210_0, W0_100);
        W0_101 = fma(kc0_110, R211_0, W0_101);
        W0_110 = fma(kc0_110, R220_0, W0_110);
        W0_200 = fma(kc0_110, R310_0, W0_200);
        const T kc1_000 = kEy0;
        W1_000 = fma(kc1_000, R000_0, W1_000);
        W1_001 = fma(kc1_000, R001_0, W1_001);
        W1_002 = fma(kc1_000, R002_0, W1_002);
        W1_010 = fma(kc1_000, R010_0, W1_010);
        W1_011 = fma(kc1_000, R011_0, W1_011);
        W1_020 = fma(kc1_000, R020_0, W1_020);
        W1_100 = fma(kc1_000, R100_0, W1_100);
        W1_101 = fma(kc1_000, R101_0, W1_101);
        W1_110 = fma(kc1_000, R110_0, W1_110);
        W1_200 = fma(kc1_000, R200_0, W1_200);
        const T kc1_010 = -kEy1;
        W1_000 = fma(kc1_010, R010_0, W1_000);
        W1_001 = fma(kc1_010, R011_0, W1_001);
        W1_002 = fma(kc1_010, R012_0, W1_002);
        W1_010 = fma(kc1_010, R020_0, W1_010);
        W1_011 = fma(kc1_010, R021_0, W1_011);
        W1_020 = fma(kc1_010, R030_0, W1_020);
        W1_100 = fma(kc1_010, R110_0, W1_100);
        W1_101 = fma(kc1_010, R111_0, W1_101);
        W1_110 = fma(kc1_010, R120_0, W1_110);
        W1_200 = fma(kc1_010, R210_0, W1_200);
        const T kc1_020 = kh2;
        W1_000 = fma(kc1_020, R020_0, W1_000);
        W1_001 = fma(kc1_020, R021_0, W1_001);
        W1_002 = fma(kc1_020, R022_0, W1_002);
        W1_010 = fma(kc1_020, R030_0, W1_010);
        W1_011 = fma(kc1_020, R031_0, W1_011);
        W1_020 = fma(kc1_020, R040_0, W1_020);
        W1_100 = fma(kc1_020, R120_0, W1_100);
        W1_101 = fma(kc1_020, R121_0, W1_101);
        W1_110 = fma(kc1_020, R130_0, W1_110);
        W1_200 = fma(kc1_020, R220_0, W1_200);
        const T kc2_000 = kAy * kBz;
        W2_000 = fma(kc2_000, R000_0, W2_000);
        W2_001 = fma(kc2_000, R001_0, W2_001);
        W2_002 = fma(kc2_000, R002_0, W2_002);
        W2_010 = fma(kc2_000, R010_0, W2_010);
        W2_011 = fma(kc2_000, R011_0, W2_011);
        W2_020 = fma(kc2_000, R020_0, W2_020);
        W2_100 = fma(kc2_000, R100_0, W2_100);
        W2_101 = fma(kc2_000, R101_0, W2_101);
        W2_110 = fma(kc2_000, R110_0, W2_110);
        W2_200 = fma(kc2_000, R200_0, W2_200);
        const T kc2_001 = -kAy * kh;
        W2_000 = fma(kc2_001, R001_0, W2_000);
        W2_001 = fma(kc2_001, R002_0, W2_001);
        W2_002 = fma(kc2_001, R003_0, W2_002);
        W2_010 = fma(kc2_001, R011_0, W2_010);
        W2_011 = fma(kc2_001, R012_0, W2_011);
        W2_020 = fma(kc2_001, R021_0, W2_020);
        W2_100 = fma(kc2_001, R101_0, W2_100);
        W2_101 = fma(kc2_001, R102_0, W2_101);
        W2_110 = fma(kc2_001, R111_0, W2_110);
        W2_200 = fma(kc2_001, R201_0, W2_200);
        const T kc2_010 = -kh * kBz;
        W2_000 = fma(kc2_010, R010_0, W2_000);
        W2_001 = fma(kc2_010, R011_0, W2_001);
        W2_002 = fma(kc2_010, R012_0, W2_002);
        W2_010 = fma(kc2_010, R020_0, W2_010);
        W2_011 = fma(kc2_010, R021_0, W2_011);
        W2_020 = fma(kc2_010, R030_0, W2_020);
        W2_100 = fma(kc2_010, R110_0, W2_100);
        W2_101 = fma(kc2_010, R111_0, W2_101);
        W2_110 = fma(kc2_010, R120_0, W2_110);
        W2_200 = fma(kc2_010, R210_0, W2_200);
        const T kc2_011 = kh * kh;
        W2_000 = fma(kc2_011, R011_0, W2_000);
        W2_001 = fma(kc2_011, R012_0, W2_001);
        W2_002 = fma(kc2_011, R013_0, W2_002);
        W2_010 = fma(kc2_011, R021_0, W2_010);
        W2_011 = fma(kc2_011, R022_0, W2_011);
        W2_020 = fma(kc2_011, R031_0, W2_020);
        W2_100 = fma(kc2_011, R111_0, W2_100);
        W2_101 = fma(kc2_011, R112_0, W2_101);
        W2_110 = fma(kc2_011, R121_0, W2_110);
        W2_200 = fma(kc2_011, R211_0, W2_200);
      }
      const T bh = __ldg(brec + 5 * bra_fs);
      const T bAx = __ldg(brec + 6 * bra_fs);
      const T bAy = __ldg(brec + 7 * bra_fs);
      const T bAz = __ldg(brec + 8 * bra_fs);
      const T bBx = __ldg(brec + 9 * bra_fs);
      const T bBy = __ldg(brec + 10 * bra_fs);
      const T bBz = __ldg(brec + 11 * bra_fs);
      const T bEx0 = bAx * bBx + bh;
      const T bEx1 = bh * (bAx + bBx);
      const T bEy0 = bAy * bBy + bh;
      const T bEy1 = bh * (bAy + bBy);
      const T bEz0 = bAz * bBz + bh;
      const T bEz1 = bh * (bAz + bBz);
      const T bh2 = bh * bh;
      I[0] = fma(bEx0, W0_000, I[0]);
      I[0] = fma(bEx1, W0_100, I[0]);
      I[0] = fma(bh2, W0_200, I[0]);
      I[1] = fma(bEx0, W1_000, I[1]);
      I[1] = fma(bEx1, W1_100, I[1]);
      I[1] = fma(bh2, W1_200, I[1]);
      I[2] = fma(bEx0, W2_000, I[2]);
      I[2] = fma(bEx1, W2_100, I[2]);
      I[2] = fma(bh2, W2_200, I[2]);
      I[3] = fma(bAx * bBy, W0_000, I[3]);
      I[3] = fma(bAx * bh, W0_010, I[3]);
      I[3] = fma(bh * bBy, W0_100, I[3]);
      I[3] = fma(bh * bh, W0_110, I[3]);
      I[4] = fma(bAx * bBy, W1_000, I[4]);
      I[4] = fma(bAx * bh, W1_010, I[4]);
      I[4] = fma(bh * bBy, W1_100, I[4]);
      I[4] = fma(bh * bh, W1_110, I[4]);
      I[5] = fma(bAx * bBy, W2_000, I[5]);
      I[5] = fma(bAx * bh, W2_010, I[5]);
      I[5] = fma(bh * bBy, W2_100, I[5]);
      I[5] = fma(bh * bh, W2_110, I[5]);
      I[6] = fma(bAx * bBz, W0_000, I[6]);
      I[6] = fma(bAx * bh, W0_001, I[6]);
      I[6] = fma(bh * bBz, W0_100, I[6]);
      I[6] = fma(bh * bh, W0_101, I[6]);
      I[7] = fma(bAx * bBz, W1_000, I[7]);
      I[7] = fma(bAx * bh, W1_001, I[7]);
      I[7] = fma(bh * bBz, W1_100, I[7]);
      I[7] = fma(bh * bh, W1_101, I[7]);
      I[8] = fma(bAx * bBz, W2_000, I[8]);
      I[8] = fma(bAx * bh, W2_001, I[8]);
      I[8] = fma(bh * bBz, W2_100, I[8]);
      I[8] = fma(bh * bh, W2_101, I[8]);
      I[9] = fma(bBx * bAy, W0_000, I[9]);
      I[9] = fma(bBx * bh, W0_010, I[9]);
      I[9] = fma(bh * bAy, W0_100, I[9]);
      I[9] = fma(bh * bh, W0_110, I[9]);
      I[10] = fma(bBx * bAy, W1_000, I[10]);
      I[10] = fma(bBx * bh, W1_010, I[10]);
      I[10] = fma(bh * bAy, W1_100, I[10]);
      I[10] = fma(bh * bh, W1_110, I[10]);
      I[11] = fma(bBx * bAy, W2_000, I[11]);
      I[11] = fma(bBx * bh, W2_010, I[11]);
      I[11] = fma(bh * bAy, W2_100, I[11]);
      I[11] = fma(bh * bh, W2_110, I[11]);
      I[12] = fma(bEy0, W0_000, I[12]);
      I[12] = fma(bEy1, W0_010, I[12]);
      I[12] = fma(bh2, W0_020, I[12]);
      I[13] = fma(bEy0, W1_000, I[13]);
      I[13] = fma(bEy1, W1_010, I[13]);
      I[13] = fma(bh2, W1_020, I[13]);
      I[14] = fma(bEy0, W2_000, I[14]);
      I[14] = fma(bEy1, W2_010, I[14]);
      I[14] = fma(bh2, W2_020, I[14]);
      I[15] = fma(bAy * bBz, W0_000, I[15]);
      I[15] = fma(bAy * bh, W0_001, I[15]);
      I[15] = fma(bh * bBz, W0_010, I[15]);
      I[15] = fma(bh * bh, W0_011, I[15]);
      I[16] = fma(bAy * bBz, W1_000, I[16]);
      I[16] = fma(bAy * bh, W1_001, I[16]);
      I[16] = fma(bh * bBz, W1_010, I[16]);
      I[16] = fma(bh * bh, W1_011, I[16]);
      I[17] = fma(bAy * bBz, W2_000, I[17]);
      I[17] = fma(bAy * bh, W2_001, I[17]);
      I[17] = fma(bh * bBz, W2_010, I[17]);
      I[17] = fma(bh * bh, W2_011, I[17]);
      I[18] = fma(bBx * bAz, W0_000, I[18]);
      I[18] = fma(bBx * bh, W0_001, I[18]);
      I[18] = fma(bh * bAz, W0_100, I[18]);
      I[18] = fma(bh * bh, W0_101, I[18]);
      I[19] = fma(bBx * bAz, W1_000, I[19]);
      I[19] = fma(bBx * bh, W1_001, I[19]);
      I[19] = fma(bh * bAz, W1_100, I[19]);
      I[19] = fma(bh * bh, W1_101, I[19]);
      I[20] = fma(bBx * bAz, W2_000, I[20]);
      I[20] = fma(bBx * bh, W2_001, I[20]);
      I[20] = fma(bh * bAz, W2_100, I[20]);
      I[20] = fma(bh * bh, W2_101, I[20]);
      I[21] = fma(bBy * bAz, W0_000, I[21]);
      I[21] = fma(bBy * bh, W0_001, I[21]);
      I[21] = fma(bh * bAz, W0_010, I[21]);
      I[21] = fma(bh * bh, W0_011, I[21]);
      I[22] = fma(bBy * bAz, W1_000, I[22]);
      I[22] = fma(bBy * bh, W1_001, I[22]);
      I[22] = fma(bh * bAz, W1_010, I[22]);
      I[22] = fma(bh * bh, W1_011, I[22]);
      I[23] = fma(bBy * bAz, W2_000, I[23]);
      I[23] = fma(bBy * bh, W2_001, I[23]);
      I[23] = fma(bh * bAz, W2_010, I[23]);
      I[23] = fma(bh * bh, W2_011, I[23]);
      I[24] = fma(bEz0, W0_000, I[24]);
      I[24] = fma(bEz1, W0_001, I[24]);
      I[24] = fma(bh2, W0_002, I[24]);
      I[25] = fma(bEz0, W1_000, I[25]);
      I[25] = fma(bEz1, W1_001, I[25]);
      I[25] = fma(bh2, W1_002, I[25]);
      I[26] = fma(bEz0, W2_000, I[26]);
      I[26] = fma(bEz1, W2_001, I[26]);
      I[26] = fma(bh2, W2_002, I[26]);
    }
    return evaluated;
  }
};

// class 5: (pp|pp), split 2 of 3, bra primitives outside
template <typename T>
struct EriClass<T, 5, 2> {
  static constexpr int LA = 1, LB = 1, LC = 1, LD = 1, L = 4;
  static constexpr int NA = 3, NB = 3, NC = 3, ND = 3;
  static constexpr int NSPLIT = 3, NCD = 3, NI = 27;
  static constexpr int BRA_CLASS = 2, KET_CLASS = 2;
  __device__ static constexpr int cd_c(int m) { constexpr int v[] = {2, 2, 2}; return v[m]; }
  __device__ static constexpr int cd_d(int m) { constexpr int v[] = {0, 1, 2}; return v[m]; }
  // Returns the number of primitive quartets evaluated: both sides'
  // primitive pairs come sorted by descending primitive Schwarz factor q,
  // and the loops stop once q_bra * q_ket < eps (each skipped primitive
  // quartet is bounded by that product, Cauchy-Schwarz per primitive pair).
  __device__ __forceinline__ static int run(
      const T* __restrict__ bra, const float* __restrict__ bra_q, long long bra_stride, int bra_kmax,
      int bra_row, int bra_n,
      const T* __restrict__ ket, const float* __restrict__ ket_q, long long ket_stride, int ket_kmax,
      int ket_row, int ket_n, float eps, T (&I)[NI]) {
    #pragma unroll
    for (int q = 0; q < NI; ++q) I[q] = T(0);
    int evaluated = 0;
    const int bra_st = (int)bra_stride, ket_st = (int)ket_stride;
    const int bra_fs = bra_kmax * bra_st, ket_fs = ket_kmax * ket_st;
    const T* __restrict__ bra_p = bra + bra_row;
    const T* __restrict__ ket_p = ket + ket_row;
    const float* __restrict__ bra_qp = bra_q + bra_row;
    const float* __restrict__ ket_qp = ket_q + ket_row;
    const float kq0 = ket_qp[0];
    #pragma unroll 1
    for (int i = 0; i < bra_n; ++i) {
      const float qo = __ldg(bra_qp + i * bra_st);
      if (qo * kq0 < eps) break;
      const T* __restrict__ brec = bra_p + i * bra_st;
      const T bPx = __ldg(brec + 0);
      const T bPy = __ldg(brec + bra_fs);
      const T bPz = __ldg(brec + 2 * bra_fs);
      const T bp = __ldg(brec + 3 * bra_fs);
      const T bK = __ldg(brec + 4 * bra_fs);
      T W0_000 = T(0), W0_001 = T(0), W0_002 = T(0), W0_010 = T(0), W0_011 = T(0), W0_020 = T(0), W0_100 = T(0), W0_101 = T(0), W0_110 = T(0), W0_200 = T(0);
      T W1_000 = T(0), W1_001 = T(0), W1_002 = T(0), W1_010 = T(0), W1_011 = T(0), W1_020 = T(0), W1_100 = T(0), W1_101 = T(0), W1_110 = T(0), W1_200 = T(0);
      T W2_000 = T(0), W2_001 = T(0), W2_002 = T(0), W2_010 = T(0), W2_011 = T(0), W2_020 = T(0), W2_100 = T(0), W2_101 = T(0), W2_110 = T(0), W2_200 = T(0);
      float knq = __ldg(ket_qp);
      T knPx = __ldg(ket_p + 0), knPy = __ldg(ket_p + ket_fs), knPz = __ldg(ket_p + 2 * ket_fs), knp = __ldg(ket_p + 3 * ket_fs), knK = __ldg(ket_p + 4 * ket_fs), knh = __ldg(ket_p + 5 * ket_fs), knAx = __ldg(ket_p + 6 * ket_fs), knAy = __ldg(ket_p + 7 * ket_fs), knAz = __ldg(ket_p + 8 * ket_fs), knBx = __ldg(ket_p + 9 * ket_fs), knBy = __ldg(ket_p + 10 * ket_fs), knBz = __ldg(ket_p + 11 * ket_fs);
      #pragma unroll 1
      for (int j = 0; j < ket_n; ++j) {
        const float kcq = knq;
        const T kPx = knPx, kPy = knPy, kPz = knPz, kp = knp, kK = knK, kh = knh, kAx = knAx, kAy = knAy, kAz = knAz, kBx = knBx, kBy = knBy, kBz = knBz;
        if (qo * kcq < eps) break;
        const int jn = j + 1 < ket_n ? j + 1 : j;
        knq = __ldg(ket_qp + jn * ket_st);
        const T* __restrict__ knrec = ket_p + jn * ket_st;
        knPx = __ldg(knrec + 0);
        knPy = __ldg(knrec + ket_fs);
        knPz = __ldg(knrec + 2 * ket_fs);
        knp = __ldg(knrec + 3 * ket_fs);
        knK = __ldg(knrec + 4 * ket_fs);
        knh = __ldg(knrec + 5 * ket_fs);
        knAx = __ldg(knrec + 6 * ket_fs);
        knAy = __ldg(knrec + 7 * ket_fs);
        knAz = __ldg(knrec + 8 * ket_fs);
        knBx = __ldg(knrec + 9 * ket_fs);
        knBy = __ldg(knrec + 10 * ket_fs);
        knBz = __ldg(knrec + 11 * ket_fs);
        ++evaluated;
        const T kEx0 = kAx * kBx + kh;
        const T kEx1 = kh * (kAx + kBx);
        const T kEy0 = kAy * kBy + kh;
        const T kEy1 = kh * (kAy + kBy);
        const T kEz0 = kAz * kBz + kh;
        const T kEz1 = kh * (kAz + kBz);
        const T kh2 = kh * kh;
        const T s = bp + kp;
        const T rs = Math<T>::rsqrt(s);
        const T rho = bp * kp * (rs * rs);
        const T X = bPx - kPx, Y = bPy - kPy, Z = bPz - kPz;
        const T pre = bK * kK * rs;
        const T m2rho = T(-2) * rho;
        T F[5];
        Boys<T, 4>::eval(rho * (X * X + Y * Y + Z * Z), F);
        T cpow = pre;
        const T R000_0 = cpow * F[0];
        cpow *= m2rho;
        const T R000_1 = cpow * F[1];
        cpow *= m2rho;
        const T R000_2 = cpow * F[2];
        cpow *= m2rho;
        const T R000_3 = cpow * F[3];
        cpow *= m2rho;
        const T R000_4 = cpow * F[4];
        const T R001_3 = Z * R000_4;
        const T R001_2 = Z * R000_3;
        const T R010_2 = Y * R000_3;
        const T R100_2 = X * R000_3;
        const T R001_1 = Z * R000_2;
        const T R010_1 = Y * R000_2;
        const T R100_1 = X * R000_2;
        const T R001_0 = Z * R000_1;
        const T R010_0 = Y * R000_1;
        const T R100_0 = X * R000_1;
        const T R002_2 = Z * R001_3 + T(1) * R000_3;
        const T R011_2 = Y * R001_3;
        const T R101_2 = X * R001_3;
        const T R002_1 = Z * R001_2 + T(1) * R000_2;
        const T R011_1 = Y * R001_2;
        const T R020_1 = Y * R010_2 + T(1) * R000_2;
        const T R101_1 = X * R001_2;
        const T R110_1 = X * R010_2;
        const T R200_1 = X * R100_2 + T(1) * R000_2;
        const T R002_0 = Z * R001_1 + T(1) * R000_1;
        const T R011_0 = Y * R001_1;
        const T R020_0 = Y * R010_1 + T(1) * R000_1;
        const T R101_0 = X * R001_1;
        const T R110_0 = X * R010_1;
        const T R200_0 = X * R100_1 + T(1) * R000_1;
        const T R003_1 = Z * R002_2 + T(2) * R001_2;
        const T R012_1 = Y * R002_2;
        const T R021_1 = Y * R011_2 + T(1) * R001_2;
        const T R102_1 = X * R002_2;
        const T R111_1 = X * R011_2;
        const T R201_1 = X * R101_2 + T(1) * R001_2;
        const T R003_0 = Z * R002_1 + T(2) * R001_1;
        const T R012_0 = Y * R002_1;
        const T R021_0 = Y * R011_1 + T(1) * R001_1;
        const T R030_0 = Y * R020_1 + T(2) * R010_1;
        const T R102_0 = X * R002_1;
        const T R111_0 = X * R011_1;
        const T R120_0 = X * R020_1;
        const T R201_0 = X * R101_1 + T(1) * R001_1;
        const T R210_0 = X * R110_1 + T(1) * R010_1;
        const T R300_0 = X * R200_1 + T(2) * R100_1;
        const T R004_0 = Z * R003_1 + T(3) * R002_1;
        const T R013_0 = Y * R003_1;
        const T R022_0 = Y * R012_1 + T(1) * R002_1;
        const T R031_0 = Y * R021_1 + T(2) * R011_1;
        const T R103_0 = X * R003_1;
        const T R112_0 = X * R012_1;
        const T R121_0 = X * R021_1;
        const T R202_0 = X * R102_1 + T(1) * R002_1;
        const T R211_0 = X * R111_1 + T(1) * R011_1;
        const T R301_0 = X * R201_1 + T(2) * R101_1;
        const T kc0_000 = kBx * kAz;
        W0_000 = fma(kc0_000, R000_0, W0_000);
        W0_001 = fma(kc0_000, R001_0, W0_001);
        W0_002 = fma(kc0_000, R002_0, W0_002);
        W0_010 = fma(kc0_000, R010_0, W0_010);
        W0_011 = fma(kc0_000, R011_0, W0_011);
        W0_020 = fma(kc0_000, R020_0, W0_020);
        W0_100 = fma(kc0_000, R100_0, W0_100);
        W0_101 = fma(kc0_000, R101_0, W0_101);
        W0_110 = fma(kc0_000, R110_0, W0_110);
        W0_200 = fma(kc0_000, R200_0, W0_200);
        const T kc0_001 = -kBx * kh;
        W0_000 = fma(kc0_001, R001_0, W0_000);
        W0_001 = fma(kc0_001, R002_0, W0_001);
        W0_002 = fma(kc0_001, R003_0, W0_002);
        W0_010 = fma(kc0_001, R011_0, W0_010);
        W0_011 = fma(kc0_001, R012_0, W0_011);
        W0_020 = fma(kc0_001, R021_0, W0_020);
        W0_100 = fma(kc0_001, R101_0, W0_100);
        W0_101 = fma(kc0_001, R102_0, W0_101);
        W0_110 = fma(kc0_001, R111_0, W0_110);
        W0_200 = fma(kc0_001, R201_0, W0_200);
        const T kc0_100 = -kh * kAz;
        W0_000 = fma(kc0_100, R100_0, W0_000);
        W0_001 = fma(kc0_100, R101_0, W0_001);
        W0_002 = fma(kc0_100, R102_0, W0_002);
        W0_010 = fma(kc0_100, R110_0, W0_010);
        W0_011 = fma(kc0_100, R111_0, W0_011);
        W0_020 = fma(kc0_100, R120_0, W0_020);
        W0_100 = fma(kc0_100, R200_0, W0_100);
        W0_101 = fma(kc0_100, R201_0, W0_101);
        W0_110 = fma(kc0_100, R210_0, W0_110);
        W0_200 = fma(kc0_100, R300_0, W0_200);
        const T kc0_101 = kh * kh;
        W0_000 = fma(kc0_101, R101_0, W0_000);
        W0_001 = fma(kc0_101, R102_0, W0_001);
        W0_002 = fma(kc0_101, R103_0, W0_002);
        W0_010 = fma(kc0_101, R111_0, W0_010);
        W0_011 = fma(kc0_101, R112_0, W0_011);
        W0_020 = fma(kc0_101, R121_0, W0_020);
        W0_100 = fma(kc0_101, R201_0, W0_100);
        W0_101 = fma(kc0_101, R202_0, W0_101);
        W0_110 = fma(kc0_101, R211_0, W0_110);
        W0_200 = fma(kc0_101, R301_0, W0_200);
        const T kc1_000 = kBy * kAz;
        W1_000 = fma(kc1_000, R000_0, W1_000);
        W1_001 = fma(kc1_000, R001_0, W1_001);
        W1_002 = fma(kc1_000, R002_0, W1_002);
        W1_010 = fma(kc1_000, R010_0, W1_010);
        W1_011 = fma(kc1_000, R011_0, W1_011);
        W1_020 = fma(kc1_000, R020_0, W1_020);
        W1_100 = fma(kc1_000, R100_0, W1_100);
        W1_101 = fma(kc1_000, R101_0, W1_101);
        W1_110 = fma(kc1_000, R110_0, W1_110);
        W1_200 = fma(kc1_000, R200_0, W1_200);
        const T kc1_001 = -kBy * kh;
        W1_000 = fma(kc1_001, R001_0, W1_000);
        W1_001 = fma(kc1_001, R002_0, W1_001);
        W1_002 = fma(kc1_001, R003_0, W1_002);
        W1_010 = fma(kc1_001, R011_0, W1_010);
        W1_011 = fma(kc1_001, R012_0, W1_011);
        W1_020 = fma(kc1_001, R021_0, W1_020);
        W1_100 = fma(kc1_001, R101_0, W1_100);
        W1_101 = fma(kc1_001, R102_0, W1_101);
        W1_110 = fma(kc1_001, R111_0, W1_110);
        W1_200 = fma(kc1_001, R201_0, W1_200);
        const T kc1_010 = -kh * kAz;
        W1_000 = fma(kc1_010, R010_0, W1_000);
        W1_001 = fma(kc1_010, R011_0, W1_001);
        W1_002 = fma(kc1_010, R012_0, W1_002);
        W1_010 = fma(kc1_010, R020_0, W1_010);
        W1_011 = fma(kc1_010, R021_0, W1_011);
        W1_020 = fma(kc1_010, R030_0, W1_020);
        W1_100 = fma(kc1_010, R110_0, W1_100);
        W1_101 = fma(kc1_010, R111_0, W1_101);
        W1_110 = fma(kc1_010, R120_0, W1_110);
        W1_200 = fma(kc1_010, R210_0, W1_200);
        const T kc1_011 = kh * kh;
        W1_000 = fma(kc1_011, R011_0, W1_000);
        W1_001 = fma(kc1_011, R012_0, W1_001);
        W1_002 = fma(kc1_011, R013_0, W1_002);
        W1_010 = fma(kc1_011, R021_0, W1_010);
        W1_011 = fma(kc1_011, R022_0, W1_011);
        W1_020 = fma(kc1_011, R031_0, W1_020);
        W1_100 = fma(kc1_011, R111_0, W1_100);
        W1_101 = fma(kc1_011, R112_0, W1_101);
        W1_110 = fma(kc1_011, R121_0, W1_110);
        W1_200 = fma(kc1_011, R211_0, W1_200);
        const T kc2_000 = kEz0;
        W2_000 = fma(kc2_000, R000_0, W2_000);
        W2_001 = fma(kc2_000, R001_0, W2_001);
        W2_002 = fma(kc2_000, R002_0, W2_002);
        W2_010 = fma(kc2_000, R010_0, W2_010);
        W2_011 = fma(kc2_000, R011_0, W2_011);
        W2_020 = fma(kc2_000, R020_0, W2_020);
        W2_100 = fma(kc2_000, R100_0, W2_100);
        W2_101 = fma(kc2_000, R101_0, W2_101);
        W2_110 = fma(kc2_000, R110_0, W2_110);
        W2_200 = fma(kc2_000, R200_0, W2_200);
        const T kc2_001 = -kEz1;
        W2_000 = fma(kc2_001, R001_0, W2_000);
        W2_001 = fma(kc2_001, R002_0, W2_001);
        W2_002 = fma(kc2_001, R003_0, W2_002);
        W2_010 = fma(kc2_001, R011_0, W2_010);
        W2_011 = fma(kc2_001, R012_0, W2_011);
        W2_020 = fma(kc2_001, R021_0, W2_020);
        W2_100 = fma(kc2_001, R101_0, W2_100);
        W2_101 = fma(kc2_001, R102_0, W2_101);
        W2_110 = fma(kc2_001, R111_0, W2_110);
        W2_200 = fma(kc2_001, R201_0, W2_200);
        const T kc2_002 = kh2;
        W2_000 = fma(kc2_002, R002_0, W2_000);
        W2_001 = fma(kc2_002, R003_0, W2_001);
        W2_002 = fma(kc2_002, R004_0, W2_002);
        W2_010 = fma(kc2_002, R012_0, W2_010);
        W2_011 = fma(kc2_002, R013_0, W2_011);
        W2_020 = fma(kc2_002, R022_0, W2_020);
        W2_100 = fma(kc2_002, R102_0, W2_100);
        W2_101 = fma(kc2_002, R103_0, W2_101);
        W2_110 = fma(kc2_002, R112_0, W2_110);
        W2_200 = fma(kc2_002, R202_0, W2_200);
      }
      const T bh = __ldg(brec + 5 * bra_fs);
      const T bAx = __ldg(brec + 6 * bra_fs);
      const T bAy = __ldg(brec + 7 * bra_fs);
      const T bAz = __ldg(brec + 8 * bra_fs);
      const T bBx = __ldg(brec + 9 * bra_fs);
      const T bBy = __ldg(brec + 10 * bra_fs);
      const T bBz = __ldg(brec + 11 * bra_fs);
      const T bEx0 = bAx * bBx + bh;
      const T bEx1 = bh * (bAx + bBx);
      const T bEy0 = bAy * bBy + bh;
      const T bEy1 = bh * (bAy + bBy);
      const T bEz0 = bAz * bBz + bh;
      const T bEz1 = bh * (bAz + bBz);
      const T bh2 = bh * bh;
      I[0] = fma(bEx0, W0_000, I[0]);
      I[0] = fma(bEx1, W0_100, I[0]);
      I[0] = fma(bh2, W0_200, I[0]);
      I[1] = fma(bEx0, W1_000, I[1]);
      I[1] = fma(bEx1, W1_100, I[1]);
      I[1] = fma(bh2, W1_200, I[1]);
      I[2] = fma(bEx0, W2_000, I[2]);
      I[2] = fma(bEx1, W2_100, I[2]);
      I[2] = fma(bh2, W2_200, I[2]);
      I[3] = fma(bAx * bBy, W0_000, I[3]);
      I[3] = fma(bAx * bh, W0_010, I[3]);
      I[3] = fma(bh * bBy, W0_100, I[3]);
      I[3] = fma(bh * bh, W0_110, I[3]);
      I[4] = fma(bAx * bBy, W1_000, I[4]);
      I[4] = fma(bAx * bh, W1_010, I[4]);
      I[4] = fma(bh * bBy, W1_100, I[4]);
      I[4] = fma(bh * bh, W1_110, I[4]);
      I[5] = fma(bAx * bBy, W2_000, I[5]);
      I[5] = fma(bAx * bh, W2_010, I[5]);
      I[5] = fma(bh * bBy, W2_100, I[5]);
      I[5] = fma(bh * bh, W2_110, I[5]);
      I[6] = fma(bAx * bBz, W0_000, I[6]);
      I[6] = fma(bAx * bh, W0_001, I[6]);
      I[6] = fma(bh * bBz, W0_100, I[6]);
      I[6] = fma(bh * bh, W0_101, I[6]);
      I[7] = fma(bAx * bBz, W1_000, I[7]);
      I[7] = fma(bAx * bh, W1_001, I[7]);
      I[7] = fma(bh * bBz, W1_100, I[7]);
      I[7] = fma(bh * bh, W1_101, I[7]);
      I[8] = fma(bAx * bBz, W2_000, I[8]);
      I[8] = fma(bAx * bh, W2_001, I[8]);
      I[8] = fma(bh * bBz, W2_100, I[8]);
      I[8] = fma(bh * bh, W2_101, I[8]);
      I[9] = fma(bBx * bAy, W0_000, I[9]);
      I[9] = fma(bBx * bh, W0_010, I[9]);
      I[9] = fma(bh * bAy, W0_100, I[9]);
      I[9] = fma(bh * bh, W0_110, I[9]);
      I[10] = fma(bBx * bAy, W1_000, I[10]);
      I[10] = fma(bBx * bh, W1_010, I[10]);
      I[10] = fma(bh * bAy, W1_100, I[10]);
      I[10] = fma(bh * bh, W1_110, I[10]);
      I[11] = fma(bBx * bAy, W2_000, I[11]);
      I[11] = fma(bBx * bh, W2_010, I[11]);
      I[11] = fma(bh * bAy, W2_100, I[11]);
      I[11] = fma(bh * bh, W2_110, I[11]);
      I[12] = fma(bEy0, W0_000, I[12]);
      I[12] = fma(bEy1, W0_010, I[12]);
      I[12] = fma(bh2, W0_020, I[12]);
      I[13] = fma(bEy0, W1_000, I[13]);
      I[13] = fma(bEy1, W1_010, I[13]);
      I[13] = fma(bh2, W1_020, I[13]);
      I[14] = fma(bEy0, W2_000, I[14]);
      I[14] = fma(bEy1, W2_010, I[14]);
      I[14] = fma(bh2, W2_020, I[14]);
      I[15] = fma(bAy * bBz, W0_000, I[15]);
      I[15] = fma(bAy * bh, W0_001, I[15]);
      I[15] = fma(bh * bBz, W0_010, I[15]);
      I[15] = fma(bh * bh, W0_011, I[15]);
      I[16] = fma(bAy * bBz, W1_000, I[16]);
      I[16] = fma(bAy * bh, W1_001, I[16]);
      I[16] = fma(bh * bBz, W1_010, I[16]);
      I[16] = fma(bh * bh, W1_011, I[16]);
      I[17] = fma(bAy * bBz, W2_000, I[17]);
      I[17] = fma(bAy * bh, W2_001, I[17]);
      I[17] = fma(bh * bBz, W2_010, I[17]);
      I[17] = fma(bh * bh, W2_011, I[17]);
      I[18] = fma(bBx * bAz, W0_000, I[18]);
      I[18] = fma(bBx * bh, W0_001, I[18]);
      I[18] = fma(bh * bAz, W0_100, I[18]);
      I[18] = fma(bh * bh, W0_101, I[18]);
      I[19] = fma(bBx * bAz, W1_000, I[19]);
      I[19] = fma(bBx * bh, W1_001, I[19]);
      I[19] = fma(bh * bAz, W1_100, I[19]);
      I[19] = fma(bh * bh, W1_101, I[19]);
      I[20] = fma(bBx * bAz, W2_000, I[20]);
      I[20] = fma(bBx * bh, W2_001, I[20]);
      I[20] = fma(bh * bAz, W2_100, I[20]);
      I[20] = fma(bh * bh, W2_101, I[20]);
      I[21] = fma(bBy * bAz, W0_000, I[21]);
      I[21] = fma(bBy * bh, W0_001, I[21]);
      I[21] = fma(bh * bAz, W0_010, I[21]);
      I[21] = fma(bh * bh, W0_011, I[21]);
      I[22] = fma(bBy * bAz, W1_000, I[22]);
      I[22] = fma(bBy * bh, W1_001, I[22]);
      I[22] = fma(bh * bAz, W1_010, I[22]);
      I[22] = fma(bh * bh, W1_011, I[22]);
      I[23] = fma(bBy * bAz, W2_000, I[23]);
      I[23] = fma(bBy * bh, W2_001, I[23]);
      I[23] = fma(bh * bAz, W2_010, I[23]);
      I[23] = fma(bh * bh, W2_011, I[23]);
      I[24] = fma(bEz0, W0_000, I[24]);
      I[24] = fma(bEz1, W0_001, I[24]);
      I[24] = fma(bh2, W0_002, I[24]);
      I[25] = fma(bEz0, W1_000, I[25]);
      I[25] = fma(bEz1, W1_001, I[25]);
      I[25] = fma(bh2, W1_002, I[25]);
      I[26] = fma(bEz0, W2_000, I[26]);
      I[26] = fma(bEz1, W2_001, I[26]);
      I[26] = fma(bh2, W2_002, I[26]);
    }
    return evaluated;
  }
};

