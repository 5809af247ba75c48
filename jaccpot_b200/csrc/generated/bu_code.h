// Generated by jaccpot_b200/_tables.py -- do not edit.
// In-place v <- B v (TR = false) or B^T v (TR = true) over degrees 1..P,
// B = B_U per degree (its non-zero entries as literals).
#pragma once
namespace jb {
template <int P, bool TR> struct BApply;
template <> struct BApply<1, false> {
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[1]; const float i1 = v[2]; const float i2 = v[3];
      v[1] = 1.0f * i0;
      v[2] = 2.0f * i2;
      v[3] = 0.5f * i1;
    }
  }
};
template <> struct BApply<1, true> {
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[1]; const float i1 = v[2]; const float i2 = v[3];
      v[1] = 1.0f * i0;
      v[2] = 0.5f * i2;
      v[3] = 2.0f * i1;
    }
  }
};
template <> struct BApply<2, false> {
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[1]; const float i1 = v[2]; const float i2 = v[3];
      v[1] = 1.0f * i0;
      v[2] = 2.0f * i2;
      v[3] = 0.5f * i1;
    }
    {
      const float i0 = v[4]; const float i1 = v[5]; const float i2 = v[6]; const float i3 = v[7]; const float i4 = v[8];
      v[4] = 0.5f * i1;
      v[5] = 2.0f * i0;
      v[6] = fmaf(3.0f, i4, -0.5f * i2);
      v[7] = 1.0f * i3;
      v[8] = fmaf(0.5f, i4, 0.25f * i2);
    }
  }
};
template <> struct BApply<2, true> {
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[1]; const float i1 = v[2]; const float i2 = v[3];
      v[1] = 1.0f * i0;
      v[2] = 0.5f * i2;
      v[3] = 2.0f * i1;
    }
    {
      const float i0 = v[4]; const float i1 = v[5]; const float i2 = v[6]; const float i3 = v[7]; const float i4 = v[8];
      v[4] = 2.0f * i1;
      v[5] = 0.5f * i0;
      v[6] = fmaf(0.25f, i4, -0.5f * i2);
      v[7] = 1.0f * i3;
      v[8] = fmaf(0.5f, i4, 3.0f * i2);
    }
  }
};
template <> struct BApply<3, false> {
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[1]; const float i1 = v[2]; const float i2 = v[3];
      v[1] = 1.0f * i0;
      v[2] = 2.0f * i2;
      v[3] = 0.5f * i1;
    }
    {
      const float i0 = v[4]; const float i1 = v[5]; const float i2 = v[6]; const float i3 = v[7]; const float i4 = v[8];
      v[4] = 0.5f * i1;
      v[5] = 2.0f * i0;
      v[6] = fmaf(3.0f, i4, -0.5f * i2);
      v[7] = 1.0f * i3;
      v[8] = fmaf(0.5f, i4, 0.25f * i2);
    }
    {
      const float i0 = v[9]; const float i1 = v[10]; const float i2 = v[11]; const float i3 = v[12]; const float i4 = v[13]; const float i5 = v[14]; const float i6 = v[15];
      v[9] = fmaf(0.25f, i2, 0.25f * i0);
      v[10] = 1.0f * i1;
      v[11] = fmaf(-0.25f, i2, 3.75f * i0);
      v[12] = fmaf(5.0f, i6, -1.0f * i4);
      v[13] = fmaf(1.25f, i5, -0.375f * i3);
      v[14] = fmaf(1.5f, i6, 0.5f * i4);
      v[15] = fmaf(0.25f, i5, 0.125f * i3);
    }
  }
};
template <> struct BApply<3, true> {
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[1]; const float i1 = v[2]; const float i2 = v[3];
      v[1] = 1.0f * i0;
      v[2] = 0.5f * i2;
      v[3] = 2.0f * i1;
    }
    {
      const float i0 = v[4]; const float i1 = v[5]; const float i2 = v[6]; const float i3 = v[7]; const float i4 = v[8];
      v[4] = 2.0f * i1;
      v[5] = 0.5f * i0;
      v[6] = fmaf(0.25f, i4, -0.5f * i2);
      v[7] = 1.0f * i3;
      v[8] = fmaf(0.5f, i4, 3.0f * i2);
    }
    {
      const float i0 = v[9]; const float i1 = v[10]; const float i2 = v[11]; const float i3 = v[12]; const float i4 = v[13]; const float i5 = v[14]; const float i6 = v[15];
      v[9] = fmaf(3.75f, i2, 0.25f * i0);
      v[10] = 1.0f * i1;
      v[11] = fmaf(-0.25f, i2, 0.25f * i0);
      v[12] = fmaf(0.125f, i6, -0.375f * i4);
      v[13] = fmaf(0.5f, i5, -1.0f * i3);
      v[14] = fmaf(0.25f, i6, 1.25f * i4);
      v[15] = fmaf(1.5f, i5, 5.0f * i3);
    }
  }
};
template <> struct BApply<4, false> {
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[1]; const float i1 = v[2]; const float i2 = v[3];
      v[1] = 1.0f * i0;
      v[2] = 2.0f * i2;
      v[3] = 0.5f * i1;
    }
    {
      const float i0 = v[4]; const float i1 = v[5]; const float i2 = v[6]; const float i3 = v[7]; const float i4 = v[8];
      v[4] = 0.5f * i1;
      v[5] = 2.0f * i0;
      v[6] = fmaf(3.0f, i4, -0.5f * i2);
      v[7] = 1.0f * i3;
      v[8] = fmaf(0.5f, i4, 0.25f * i2);
    }
    {
      const float i0 = v[9]; const float i1 = v[10]; const float i2 = v[11]; const float i3 = v[12]; const float i4 = v[13]; const float i5 = v[14]; const float i6 = v[15];
      v[9] = fmaf(0.25f, i2, 0.25f * i0);
      v[10] = 1.0f * i1;
      v[11] = fmaf(-0.25f, i2, 3.75f * i0);
      v[12] = fmaf(5.0f, i6, -1.0f * i4);
      v[13] = fmaf(1.25f, i5, -0.375f * i3);
      v[14] = fmaf(1.5f, i6, 0.5f * i4);
      v[15] = fmaf(0.25f, i5, 0.125f * i3);
    }
    {
      const float i0 = v[16]; const float i1 = v[17]; const float i2 = v[18]; const float i3 = v[19]; const float i4 = v[20]; const float i5 = v[21]; const float i6 = v[22]; const float i7 = v[23]; const float i8 = v[24];
      v[16] = fmaf(0.125f, i3, 0.125f * i1);
      v[17] = fmaf(0.5f, i2, 1.0f * i0);
      v[18] = fmaf(-0.25f, i3, 1.75f * i1);
      v[19] = fmaf(-0.5f, i2, 7.0f * i0);
      v[20] = fmaf(8.75f, i8, fmaf(-1.25f, i6, 0.375f * i4));
      v[21] = fmaf(1.75f, i7, -0.75f * i5);
      v[22] = fmaf(3.5f, i8, fmaf(0.5f, i6, -0.25f * i4));
      v[23] = fmaf(0.75f, i7, 0.25f * i5);
      v[24] = fmaf(0.125f, i8, fmaf(0.125f, i6, 0.0625f * i4));
    }
  }
};
template <> struct BApply<4, true> {
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[1]; const float i1 = v[2]; const float i2 = v[3];
      v[1] = 1.0f * i0;
      v[2] = 0.5f * i2;
      v[3] = 2.0f * i1;
    }
    {
      const float i0 = v[4]; const float i1 = v[5]; const float i2 = v[6]; const float i3 = v[7]; const float i4 = v[8];
      v[4] = 2.0f * i1;
      v[5] = 0.5f * i0;
      v[6] = fmaf(0.25f, i4, -0.5f * i2);
      v[7] = 1.0f * i3;
      v[8] = fmaf(0.5f, i4, 3.0f * i2);
    }
    {
      const float i0 = v[9]; const float i1 = v[10]; const float i2 = v[11]; const float i3 = v[12]; const float i4 = v[13]; const float i5 = v[14]; const float i6 = v[15];
      v[9] = fmaf(3.75f, i2, 0.25f * i0);
      v[10] = 1.0f * i1;
      v[11] = fmaf(-0.25f, i2, 0.25f * i0);
      v[12] = fmaf(0.125f, i6, -0.375f * i4);
      v[13] = fmaf(0.5f, i5, -1.0f * i3);
      v[14] = fmaf(0.25f, i6, 1.25f * i4);
      v[15] = fmaf(1.5f, i5, 5.0f * i3);
    }
    {
      const float i0 = v[16]; const float i1 = v[17]; const float i2 = v[18]; const float i3 = v[19]; const float i4 = v[20]; const float i5 = v[21]; const float i6 = v[22]; const float i7 = v[23]; const float i8 = v[24];
      v[16] = fmaf(7.0f, i3, 1.0f * i1);
      v[17] = fmaf(1.75f, i2, 0.125f * i0);
      v[18] = fmaf(-0.5f, i3, 0.5f * i1);
      v[19] = fmaf(-0.25f, i2, 0.125f * i0);
      v[20] = fmaf(0.0625f, i8, fmaf(-0.25f, i6, 0.375f * i4));
      v[21] = fmaf(0.25f, i7, -0.75f * i5);
      v[22] = fmaf(0.125f, i8, fmaf(0.5f, i6, -1.25f * i4));
      v[23] = fmaf(0.75f, i7, 1.75f * i5);
      v[24] = fmaf(0.125f, i8, fmaf(3.5f, i6, 8.75f * i4));
    }
  }
};
template <> struct BApply<5, false> {
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[1]; const float i1 = v[2]; const float i2 = v[3];
      v[1] = 1.0f * i0;
      v[2] = 2.0f * i2;
      v[3] = 0.5f * i1;
    }
    {
      const float i0 = v[4]; const float i1 = v[5]; const float i2 = v[6]; const float i3 = v[7]; const float i4 = v[8];
      v[4] = 0.5f * i1;
      v[5] = 2.0f * i0;
      v[6] = fmaf(3.0f, i4, -0.5f * i2);
      v[7] = 1.0f * i3;
      v[8] = fmaf(0.5f, i4, 0.25f * i2);
    }
    {
      const float i0 = v[9]; const float i1 = v[10]; const float i2 = v[11]; const float i3 = v[12]; const float i4 = v[13]; const float i5 = v[14]; const float i6 = v[15];
      v[9] = fmaf(0.25f, i2, 0.25f * i0);
      v[10] = 1.0f * i1;
      v[11] = fmaf(-0.25f, i2, 3.75f * i0);
      v[12] = fmaf(5.0f, i6, -1.0f * i4);
      v[13] = fmaf(1.25f, i5, -0.375f * i3);
      v[14] = fmaf(1.5f, i6, 0.5f * i4);
      v[15] = fmaf(0.25f, i5, 0.125f * i3);
    }
    {
      const float i0 = v[16]; const float i1 = v[17]; const float i2 = v[18]; const float i3 = v[19]; const float i4 = v[20]; const float i5 = v[21]; const float i6 = v[22]; const float i7 = v[23]; const float i8 = v[24];
      v[16] = fmaf(0.125f, i3, 0.125f * i1);
      v[17] = fmaf(0.5f, i2, 1.0f * i0);
      v[18] = fmaf(-0.25f, i3, 1.75f * i1);
      v[19] = fmaf(-0.5f, i2, 7.0f * i0);
      v[20] = fmaf(8.75f, i8, fmaf(-1.25f, i6, 0.375f * i4));
      v[21] = fmaf(1.75f, i7, -0.75f * i5);
      v[22] = fmaf(3.5f, i8, fmaf(0.5f, i6, -0.25f * i4));
      v[23] = fmaf(0.75f, i7, 0.25f * i5);
      v[24] = fmaf(0.125f, i8, fmaf(0.125f, i6, 0.0625f * i4));
    }
    {
      const float i0 = v[25]; const float i1 = v[26]; const float i2 = v[27]; const float i3 = v[28]; const float i4 = v[29]; const float i5 = v[30]; const float i6 = v[31]; const float i7 = v[32]; const float i8 = v[33]; const float i9 = v[34]; const float i10 = v[35];
      v[25] = fmaf(0.0625f, i4, fmaf(0.0625f, i2, 0.0625f * i0));
      v[26] = fmaf(0.25f, i3, 0.5f * i1);
      v[27] = fmaf(-0.1875f, i4, fmaf(0.8125f, i2, 2.8125f * i0));
      v[28] = fmaf(-0.5f, i3, 3.0f * i1);
      v[29] = fmaf(0.125f, i4, fmaf(-0.875f, i2, 13.125f * i0));
      v[30] = fmaf(15.75f, i10, fmaf(-1.75f, i8, 0.75f * i6));
      v[31] = fmaf(2.625f, i9, fmaf(-0.875f, i7, 0.3125f * i5));
      v[32] = fmaf(7.5f, i10, fmaf(0.5f, i8, -0.5f * i6));
      v[33] = fmaf(1.6875f, i9, fmaf(0.1875f, i7, -0.15625f * i5));
      v[34] = fmaf(0.625f, i10, fmaf(0.375f, i8, 0.125f * i6));
      v[35] = fmaf(0.0625f, i9, fmaf(0.0625f, i7, 0.03125f * i5));
    }
  }
};
template <> struct BApply<5, true> {
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[1]; const float i1 = v[2]; const float i2 = v[3];
      v[1] = 1.0f * i0;
      v[2] = 0.5f * i2;
      v[3] = 2.0f * i1;
    }
    {
      const float i0 = v[4]; const float i1 = v[5]; const float i2 = v[6]; const float i3 = v[7]; const float i4 = v[8];
      v[4] = 2.0f * i1;
      v[5] = 0.5f * i0;
      v[6] = fmaf(0.25f, i4, -0.5f * i2);
      v[7] = 1.0f * i3;
      v[8] = fmaf(0.5f, i4, 3.0f * i2);
    }
    {
      const float i0 = v[9]; const float i1 = v[10]; const float i2 = v[11]; const float i3 = v[12]; const float i4 = v[13]; const float i5 = v[14]; const float i6 = v[15];
      v[9] = fmaf(3.75f, i2, 0.25f * i0);
      v[10] = 1.0f * i1;
      v[11] = fmaf(-0.25f, i2, 0.25f * i0);
      v[12] = fmaf(0.125f, i6, -0.375f * i4);
      v[13] = fmaf(0.5f, i5, -1.0f * i3);
      v[14] = fmaf(0.25f, i6, 1.25f * i4);
      v[15] = fmaf(1.5f, i5, 5.0f * i3);
    }
    {
      const float i0 = v[16]; const float i1 = v[17]; const float i2 = v[18]; const float i3 = v[19]; const float i4 = v[20]; const float i5 = v[21]; const float i6 = v[22]; const float i7 = v[23]; const float i8 = v[24];
      v[16] = fmaf(7.0f, i3, 1.0f * i1);
      v[17] = fmaf(1.75f, i2, 0.125f * i0);
      v[18] = fmaf(-0.5f, i3, 0.5f * i1);
      v[19] = fmaf(-0.25f, i2, 0.125f * i0);
      v[20] = fmaf(0.0625f, i8, fmaf(-0.25f, i6, 0.375f * i4));
      v[21] = fmaf(0.25f, i7, -0.75f * i5);
      v[22] = fmaf(0.125f, i8, fmaf(0.5f, i6, -1.25f * i4));
      v[23] = fmaf(0.75f, i7, 1.75f * i5);
      v[24] = fmaf(0.125f, i8, fmaf(3.5f, i6, 8.75f * i4));
    }
    {
      const float i0 = v[25]; const float i1 = v[26]; const float i2 = v[27]; const float i3 = v[28]; const float i4 = v[29]; const float i5 = v[30]; const float i6 = v[31]; const float i7 = v[32]; const float i8 = v[33]; const float i9 = v[34]; const float i10 = v[35];
      v[25] = fmaf(13.125f, i4, fmaf(2.8125f, i2, 0.0625f * i0));
      v[26] = fmaf(3.0f, i3, 0.5f * i1);
      v[27] = fmaf(-0.875f, i4, fmaf(0.8125f, i2, 0.0625f * i0));
      v[28] = fmaf(-0.5f, i3, 0.25f * i1);
      v[29] = fmaf(0.125f, i4, fmaf(-0.1875f, i2, 0.0625f * i0));
      v[30] = fmaf(0.03125f, i10, fmaf(-0.15625f, i8, 0.3125f * i6));
      v[31] = fmaf(0.125f, i9, fmaf(-0.5f, i7, 0.75f * i5));
      v[32] = fmaf(0.0625f, i10, fmaf(0.1875f, i8, -0.875f * i6));
      v[33] = fmaf(0.375f, i9, fmaf(0.5f, i7, -1.75f * i5));
      v[34] = fmaf(0.0625f, i10, fmaf(1.6875f, i8, 2.625f * i6));
      v[35] = fmaf(0.625f, i9, fmaf(7.5f, i7, 15.75f * i5));
    }
  }
};
template <> struct BApply<6, false> {
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[1]; const float i1 = v[2]; const float i2 = v[3];
      v[1] = 1.0f * i0;
      v[2] = 2.0f * i2;
      v[3] = 0.5f * i1;
    }
    {
      const float i0 = v[4]; const float i1 = v[5]; const float i2 = v[6]; const float i3 = v[7]; const float i4 = v[8];
      v[4] = 0.5f * i1;
      v[5] = 2.0f * i0;
      v[6] = fmaf(3.0f, i4, -0.5f * i2);
      v[7] = 1.0f * i3;
      v[8] = fmaf(0.5f, i4, 0.25f * i2);
    }
    {
      const float i0 = v[9]; const float i1 = v[10]; const float i2 = v[11]; const float i3 = v[12]; const float i4 = v[13]; const float i5 = v[14]; const float i6 = v[15];
      v[9] = fmaf(0.25f, i2, 0.25f * i0);
      v[10] = 1.0f * i1;
      v[11] = fmaf(-0.25f, i2, 3.75f * i0);
      v[12] = fmaf(5.0f, i6, -1.0f * i4);
      v[13] = fmaf(1.25f, i5, -0.375f * i3);
      v[14] = fmaf(1.5f, i6, 0.5f * i4);
      v[15] = fmaf(0.25f, i5, 0.125f * i3);
    }
    {
      const float i0 = v[16]; const float i1 = v[17]; const float i2 = v[18]; const float i3 = v[19]; const float i4 = v[20]; const float i5 = v[21]; const float i6 = v[22]; const float i7 = v[23]; const float i8 = v[24];
      v[16] = fmaf(0.125f, i3, 0.125f * i1);
      v[17] = fmaf(0.5f, i2, 1.0f * i0);
      v[18] = fmaf(-0.25f, i3, 1.75f * i1);
      v[19] = fmaf(-0.5f, i2, 7.0f * i0);
      v[20] = fmaf(8.75f, i8, fmaf(-1.25f, i6, 0.375f * i4));
      v[21] = fmaf(1.75f, i7, -0.75f * i5);
      v[22] = fmaf(3.5f, i8, fmaf(0.5f, i6, -0.25f * i4));
      v[23] = fmaf(0.75f, i7, 0.25f * i5);
      v[24] = fmaf(0.125f, i8, fmaf(0.125f, i6, 0.0625f * i4));
    }
    {
      const float i0 = v[25]; const float i1 = v[26]; const float i2 = v[27]; const float i3 = v[28]; const float i4 = v[29]; const float i5 = v[30]; const float i6 = v[31]; const float i7 = v[32]; const float i8 = v[33]; const float i9 = v[34]; const float i10 = v[35];
      v[25] = fmaf(0.0625f, i4, fmaf(0.0625f, i2, 0.0625f * i0));
      v[26] = fmaf(0.25f, i3, 0.5f * i1);
      v[27] = fmaf(-0.1875f, i4, fmaf(0.8125f, i2, 2.8125f * i0));
      v[28] = fmaf(-0.5f, i3, 3.0f * i1);
      v[29] = fmaf(0.125f, i4, fmaf(-0.875f, i2, 13.125f * i0));
      v[30] = fmaf(15.75f, i10, fmaf(-1.75f, i8, 0.75f * i6));
      v[31] = fmaf(2.625f, i9, fmaf(-0.875f, i7, 0.3125f * i5));
      v[32] = fmaf(7.5f, i10, fmaf(0.5f, i8, -0.5f * i6));
      v[33] = fmaf(1.6875f, i9, fmaf(0.1875f, i7, -0.15625f * i5));
      v[34] = fmaf(0.625f, i10, fmaf(0.375f, i8, 0.125f * i6));
      v[35] = fmaf(0.0625f, i9, fmaf(0.0625f, i7, 0.03125f * i5));
    }
    {
      const float i0 = v[36]; const float i1 = v[37]; const float i2 = v[38]; const float i3 = v[39]; const float i4 = v[40]; const float i5 = v[41]; const float i6 = v[42]; const float i7 = v[43]; const float i8 = v[44]; const float i9 = v[45]; const float i10 = v[46]; const float i11 = v[47]; const float i12 = v[48];
      v[36] = fmaf(0.03125f, i5, fmaf(0.03125f, i3, 0.03125f * i1));
      v[37] = fmaf(0.125f, i4, fmaf(0.25f, i2, 0.375f * i0));
      v[38] = fmaf(-0.125f, i5, fmaf(0.375f, i3, 1.375f * i1));
      v[39] = fmaf(-0.375f, i4, fmaf(1.25f, i2, 6.875f * i0));
      v[40] = fmaf(0.15625f, i5, fmaf(-0.84375f, i3, 5.15625f * i1));
      v[41] = fmaf(0.25f, i4, fmaf(-1.5f, i2, 24.75f * i0));
      v[42] = fmaf(28.875f, i12, fmaf(-2.625f, i10, fmaf(0.875f, i8, -0.3125f * i6)));
      v[43] = fmaf(4.125f, i11, fmaf(-1.125f, i9, 0.625f * i7));
      v[44] = fmaf(15.46875f, i12, fmaf(0.46875f, i10, fmaf(-0.53125f, i8, 0.234375f * i6)));
      v[45] = fmaf(3.4375f, i11, fmaf(0.0625f, i9, -0.3125f * i7));
      v[46] = fmaf(2.0625f, i12, fmaf(0.8125f, i10, fmaf(0.0625f, i8, -0.09375f * i6)));
      v[47] = fmaf(0.3125f, i11, fmaf(0.1875f, i9, 0.0625f * i7));
      v[48] = fmaf(0.03125f, i12, fmaf(0.03125f, i10, fmaf(0.03125f, i8, 0.015625f * i6)));
    }
  }
};
template <> struct BApply<6, true> {
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[1]; const float i1 = v[2]; const float i2 = v[3];
      v[1] = 1.0f * i0;
      v[2] = 0.5f * i2;
      v[3] = 2.0f * i1;
    }
    {
      const float i0 = v[4]; const float i1 = v[5]; const float i2 = v[6]; const float i3 = v[7]; const float i4 = v[8];
      v[4] = 2.0f * i1;
      v[5] = 0.5f * i0;
      v[6] = fmaf(0.25f, i4, -0.5f * i2);
      v[7] = 1.0f * i3;
      v[8] = fmaf(0.5f, i4, 3.0f * i2);
    }
    {
      const float i0 = v[9]; const float i1 = v[10]; const float i2 = v[11]; const float i3 = v[12]; const float i4 = v[13]; const float i5 = v[14]; const float i6 = v[15];
      v[9] = fmaf(3.75f, i2, 0.25f * i0);
      v[10] = 1.0f * i1;
      v[11] = fmaf(-0.25f, i2, 0.25f * i0);
      v[12] = fmaf(0.125f, i6, -0.375f * i4);
      v[13] = fmaf(0.5f, i5, -1.0f * i3);
      v[14] = fmaf(0.25f, i6, 1.25f * i4);
      v[15] = fmaf(1.5f, i5, 5.0f * i3);
    }
    {
      const float i0 = v[16]; const float i1 = v[17]; const float i2 = v[18]; const float i3 = v[19]; const float i4 = v[20]; const float i5 = v[21]; const float i6 = v[22]; const float i7 = v[23]; const float i8 = v[24];
      v[16] = fmaf(7.0f, i3, 1.0f * i1);
      v[17] = fmaf(1.75f, i2, 0.125f * i0);
      v[18] = fmaf(-0.5f, i3, 0.5f * i1);
      v[19] = fmaf(-0.25f, i2, 0.125f * i0);
      v[20] = fmaf(0.0625f, i8, fmaf(-0.25f, i6, 0.375f * i4));
      v[21] = fmaf(0.25f, i7, -0.75f * i5);
      v[22] = fmaf(0.125f, i8, fmaf(0.5f, i6, -1.25f * i4));
      v[23] = fmaf(0.75f, i7, 1.75f * i5);
      v[24] = fmaf(0.125f, i8, fmaf(3.5f, i6, 8.75f * i4));
    }
    {
      const float i0 = v[25]; const float i1 = v[26]; const float i2 = v[27]; const float i3 = v[28]; const float i4 = v[29]; const float i5 = v[30]; const float i6 = v[31]; const float i7 = v[32]; const float i8 = v[33]; const float i9 = v[34]; const float i10 = v[35];
      v[25] = fmaf(13.125f, i4, fmaf(2.8125f, i2, 0.0625f * i0));
      v[26] = fmaf(3.0f, i3, 0.5f * i1);
      v[27] = fmaf(-0.875f, i4, fmaf(0.8125f, i2, 0.0625f * i0));
      v[28] = fmaf(-0.5f, i3, 0.25f * i1);
      v[29] = fmaf(0.125f, i4, fmaf(-0.1875f, i2, 0.0625f * i0));
      v[30] = fmaf(0.03125f, i10, fmaf(-0.15625f, i8, 0.3125f * i6));
      v[31] = fmaf(0.125f, i9, fmaf(-0.5f, i7, 0.75f * i5));
      v[32] = fmaf(0.0625f, i10, fmaf(0.1875f, i8, -0.875f * i6));
      v[33] = fmaf(0.375f, i9, fmaf(0.5f, i7, -1.75f * i5));
      v[34] = fmaf(0.0625f, i10, fmaf(1.6875f, i8, 2.625f * i6));
      v[35] = fmaf(0.625f, i9, fmaf(7.5f, i7, 15.75f * i5));
    }
    {
      const float i0 = v[36]; const float i1 = v[37]; const float i2 = v[38]; const float i3 = v[39]; const float i4 = v[40]; const float i5 = v[41]; const float i6 = v[42]; const float i7 = v[43]; const float i8 = v[44]; const float i9 = v[45]; const float i10 = v[46]; const float i11 = v[47]; const float i12 = v[48];
      v[36] = fmaf(24.75f, i5, fmaf(6.875f, i3, 0.375f * i1));
      v[37] = fmaf(5.15625f, i4, fmaf(1.375f, i2, 0.03125f * i0));
      v[38] = fmaf(-1.5f, i5, fmaf(1.25f, i3, 0.25f * i1));
      v[39] = fmaf(-0.84375f, i4, fmaf(0.375f, i2, 0.03125f * i0));
      v[40] = fmaf(0.25f, i5, fmaf(-0.375f, i3, 0.125f * i1));
      v[41] = fmaf(0.15625f, i4, fmaf(-0.125f, i2, 0.03125f * i0));
      v[42] = fmaf(0.015625f, i12, fmaf(-0.09375f, i10, fmaf(0.234375f, i8, -0.3125f * i6)));
      v[43] = fmaf(0.0625f, i11, fmaf(-0.3125f, i9, 0.625f * i7));
      v[44] = fmaf(0.03125f, i12, fmaf(0.0625f, i10, fmaf(-0.53125f, i8, 0.875f * i6)));
      v[45] = fmaf(0.1875f, i11, fmaf(0.0625f, i9, -1.125f * i7));
      v[46] = fmaf(0.03125f, i12, fmaf(0.8125f, i10, fmaf(0.46875f, i8, -2.625f * i6)));
      v[47] = fmaf(0.3125f, i11, fmaf(3.4375f, i9, 4.125f * i7));
      v[48] = fmaf(0.03125f, i12, fmaf(2.0625f, i10, fmaf(15.46875f, i8, 28.875f * i6)));
    }
  }
};
template <> struct BApply<7, false> {
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[1]; const float i1 = v[2]; const float i2 = v[3];
      v[1] = 1.0f * i0;
      v[2] = 2.0f * i2;
      v[3] = 0.5f * i1;
    }
    {
      const float i0 = v[4]; const float i1 = v[5]; const float i2 = v[6]; const float i3 = v[7]; const float i4 = v[8];
      v[4] = 0.5f * i1;
      v[5] = 2.0f * i0;
      v[6] = fmaf(3.0f, i4, -0.5f * i2);
      v[7] = 1.0f * i3;
      v[8] = fmaf(0.5f, i4, 0.25f * i2);
    }
    {
      const float i0 = v[9]; const float i1 = v[10]; const float i2 = v[11]; const float i3 = v[12]; const float i4 = v[13]; const float i5 = v[14]; const float i6 = v[15];
      v[9] = fmaf(0.25f, i2, 0.25f * i0);
      v[10] = 1.0f * i1;
      v[11] = fmaf(-0.25f, i2, 3.75f * i0);
      v[12] = fmaf(5.0f, i6, -1.0f * i4);
      v[13] = fmaf(1.25f, i5, -0.375f * i3);
      v[14] = fmaf(1.5f, i6, 0.5f * i4);
      v[15] = fmaf(0.25f, i5, 0.125f * i3);
    }
    {
      const float i0 = v[16]; const float i1 = v[17]; const float i2 = v[18]; const float i3 = v[19]; const float i4 = v[20]; const float i5 = v[21]; const float i6 = v[22]; const float i7 = v[23]; const float i8 = v[24];
      v[16] = fmaf(0.125f, i3, 0.125f * i1);
      v[17] = fmaf(0.5f, i2, 1.0f * i0);
      v[18] = fmaf(-0.25f, i3, 1.75f * i1);
      v[19] = fmaf(-0.5f, i2, 7.0f * i0);
      v[20] = fmaf(8.75f, i8, fmaf(-1.25f, i6, 0.375f * i4));
      v[21] = fmaf(1.75f, i7, -0.75f * i5);
      v[22] = fmaf(3.5f, i8, fmaf(0.5f, i6, -0.25f * i4));
      v[23] = fmaf(0.75f, i7, 0.25f * i5);
      v[24] = fmaf(0.125f, i8, fmaf(0.125f, i6, 0.0625f * i4));
    }
    {
      const float i0 = v[25]; const float i1 = v[26]; const float i2 = v[27]; const float i3 = v[28]; const float i4 = v[29]; const float i5 = v[30]; const float i6 = v[31]; const float i7 = v[32]; const float i8 = v[33]; const float i9 = v[34]; const float i10 = v[35];
      v[25] = fmaf(0.0625f, i4, fmaf(0.0625f, i2, 0.0625f * i0));
      v[26] = fmaf(0.25f, i3, 0.5f * i1);
      v[27] = fmaf(-0.1875f, i4, fmaf(0.8125f, i2, 2.8125f * i0));
      v[28] = fmaf(-0.5f, i3, 3.0f * i1);
      v[29] = fmaf(0.125f, i4, fmaf(-0.875f, i2, 13.125f * i0));
      v[30] = fmaf(15.75f, i10, fmaf(-1.75f, i8, 0.75f * i6));
      v[31] = fmaf(2.625f, i9, fmaf(-0.875f, i7, 0.3125f * i5));
      v[32] = fmaf(7.5f, i10, fmaf(0.5f, i8, -0.5f * i6));
      v[33] = fmaf(1.6875f, i9, fmaf(0.1875f, i7, -0.15625f * i5));
      v[34] = fmaf(0.625f, i10, fmaf(0.375f, i8, 0.125f * i6));
      v[35] = fmaf(0.0625f, i9, fmaf(0.0625f, i7, 0.03125f * i5));
    }
    {
      const float i0 = v[36]; const float i1 = v[37]; const float i2 = v[38]; const float i3 = v[39]; const float i4 = v[40]; const float i5 = v[41]; const float i6 = v[42]; const float i7 = v[43]; const float i8 = v[44]; const float i9 = v[45]; const float i10 = v[46]; const float i11 = v[47]; const float i12 = v[48];
      v[36] = fmaf(0.03125f, i5, fmaf(0.03125f, i3, 0.03125f * i1));
      v[37] = fmaf(0.125f, i4, fmaf(0.25f, i2, 0.375f * i0));
      v[38] = fmaf(-0.125f, i5, fmaf(0.375f, i3, 1.375f * i1));
      v[39] = fmaf(-0.375f, i4, fmaf(1.25f, i2, 6.875f * i0));
      v[40] = fmaf(0.15625f, i5, fmaf(-0.84375f, i3, 5.15625f * i1));
      v[41] = fmaf(0.25f, i4, fmaf(-1.5f, i2, 24.75f * i0));
      v[42] = fmaf(28.875f, i12, fmaf(-2.625f, i10, fmaf(0.875f, i8, -0.3125f * i6)));
      v[43] = fmaf(4.125f, i11, fmaf(-1.125f, i9, 0.625f * i7));
      v[44] = fmaf(15.46875f, i12, fmaf(0.46875f, i10, fmaf(-0.53125f, i8, 0.234375f * i6)));
      v[45] = fmaf(3.4375f, i11, fmaf(0.0625f, i9, -0.3125f * i7));
      v[46] = fmaf(2.0625f, i12, fmaf(0.8125f, i10, fmaf(0.0625f, i8, -0.09375f * i6)));
      v[47] = fmaf(0.3125f, i11, fmaf(0.1875f, i9, 0.0625f * i7));
      v[48] = fmaf(0.03125f, i12, fmaf(0.03125f, i10, fmaf(0.03125f, i8, 0.015625f * i6)));
    }
    {
      const float i0 = v[49]; const float i1 = v[50]; const float i2 = v[51]; const float i3 = v[52]; const float i4 = v[53]; const float i5 = v[54]; const float i6 = v[55]; const float i7 = v[56]; const float i8 = v[57]; const float i9 = v[58]; const float i10 = v[59]; const float i11 = v[60]; const float i12 = v[61]; const float i13 = v[62]; const float i14 = v[63];
      v[49] = fmaf(0.015625f, i6, fmaf(0.015625f, i4, fmaf(0.015625f, i2, 0.015625f * i0)));
      v[50] = fmaf(0.0625f, i5, fmaf(0.125f, i3, 0.1875f * i1));
      v[51] = fmaf(-0.078125f, i6, fmaf(0.171875f, i4, fmaf(0.671875f, i2, 1.421875f * i0)));
      v[52] = fmaf(-0.25f, i5, fmaf(0.5f, i3, 3.25f * i1));
      v[53] = fmaf(0.140625f, i6, fmaf(-0.609375f, i4, fmaf(1.890625f, i2, 15.640625f * i0)));
      v[54] = fmaf(0.3125f, i5, fmaf(-1.375f, i3, 8.9375f * i1));
      v[55] = fmaf(-0.078125f, i6, fmaf(0.421875f, i4, fmaf(-2.578125f, i2, 46.921875f * i0)));
      v[56] = fmaf(53.625f, i14, fmaf(-4.125f, i12, fmaf(1.125f, i10, -0.625f * i8)));
      v[57] = fmaf(6.703125f, i13, fmaf(-1.546875f, i11, fmaf(0.703125f, i9, -0.2734375f * i7)));
      v[58] = fmaf(31.28125f, i14, fmaf(0.34375f, i12, fmaf(-0.59375f, i10, 0.46875f * i8)));
      v[59] = fmaf(6.703125f, i13, fmaf(-0.171875f, i11, fmaf(-0.296875f, i9, 0.1640625f * i7)));
      v[60] = fmaf(5.6875f, i14, fmaf(1.5625f, i12, fmaf(-0.0625f, i10, -0.1875f * i8)));
      v[61] = fmaf(1.015625f, i13, fmaf(0.390625f, i11, fmaf(0.015625f, i9, -0.0546875f * i7)));
      v[62] = fmaf(0.21875f, i14, fmaf(0.15625f, i12, fmaf(0.09375f, i10, 0.03125f * i8)));
      v[63] = fmaf(0.015625f, i13, fmaf(0.015625f, i11, fmaf(0.015625f, i9, 0.0078125f * i7)));
    }
  }
};
template <> struct BApply<7, true> {
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[1]; const float i1 = v[2]; const float i2 = v[3];
      v[1] = 1.0f * i0;
      v[2] = 0.5f * i2;
      v[3] = 2.0f * i1;
    }
    {
      const float i0 = v[4]; const float i1 = v[5]; const float i2 = v[6]; const float i3 = v[7]; const float i4 = v[8];
      v[4] = 2.0f * i1;
      v[5] = 0.5f * i0;
      v[6] = fmaf(0.25f, i4, -0.5f * i2);
      v[7] = 1.0f * i3;
      v[8] = fmaf(0.5f, i4, 3.0f * i2);
    }
    {
      const float i0 = v[9]; const float i1 = v[10]; const float i2 = v[11]; const float i3 = v[12]; const float i4 = v[13]; const float i5 = v[14]; const float i6 = v[15];
      v[9] = fmaf(3.75f, i2, 0.25f * i0);
      v[10] = 1.0f * i1;
      v[11] = fmaf(-0.25f, i2, 0.25f * i0);
      v[12] = fmaf(0.125f, i6, -0.375f * i4);
      v[13] = fmaf(0.5f, i5, -1.0f * i3);
      v[14] = fmaf(0.25f, i6, 1.25f * i4);
      v[15] = fmaf(1.5f, i5, 5.0f * i3);
    }
    {
      const float i0 = v[16]; const float i1 = v[17]; const float i2 = v[18]; const float i3 = v[19]; const float i4 = v[20]; const float i5 = v[21]; const float i6 = v[22]; const float i7 = v[23]; const float i8 = v[24];
      v[16] = fmaf(7.0f, i3, 1.0f * i1);
      v[17] = fmaf(1.75f, i2, 0.125f * i0);
      v[18] = fmaf(-0.5f, i3, 0.5f * i1);
      v[19] = fmaf(-0.25f, i2, 0.125f * i0);
      v[20] = fmaf(0.0625f, i8, fmaf(-0.25f, i6, 0.375f * i4));
      v[21] = fmaf(0.25f, i7, -0.75f * i5);
      v[22] = fmaf(0.125f, i8, fmaf(0.5f, i6, -1.25f * i4));
      v[23] = fmaf(0.75f, i7, 1.75f * i5);
      v[24] = fmaf(0.125f, i8, fmaf(3.5f, i6, 8.75f * i4));
    }
    {
      const float i0 = v[25]; const float i1 = v[26]; const float i2 = v[27]; const float i3 = v[28]; const float i4 = v[29]; const float i5 = v[30]; const float i6 = v[31]; const float i7 = v[32]; const float i8 = v[33]; const float i9 = v[34]; const float i10 = v[35];
      v[25] = fmaf(13.125f, i4, fmaf(2.8125f, i2, 0.0625f * i0));
      v[26] = fmaf(3.0f, i3, 0.5f * i1);
      v[27] = fmaf(-0.875f, i4, fmaf(0.8125f, i2, 0.0625f * i0));
      v[28] = fmaf(-0.5f, i3, 0.25f * i1);
      v[29] = fmaf(0.125f, i4, fmaf(-0.1875f, i2, 0.0625f * i0));
      v[30] = fmaf(0.03125f, i10, fmaf(-0.15625f, i8, 0.3125f * i6));
      v[31] = fmaf(0.125f, i9, fmaf(-0.5f, i7, 0.75f * i5));
      v[32] = fmaf(0.0625f, i10, fmaf(0.1875f, i8, -0.875f * i6));
      v[33] = fmaf(0.375f, i9, fmaf(0.5f, i7, -1.75f * i5));
      v[34] = fmaf(0.0625f, i10, fmaf(1.6875f, i8, 2.625f * i6));
      v[35] = fmaf(0.625f, i9, fmaf(7.5f, i7, 15.75f * i5));
    }
    {
      const float i0 = v[36]; const float i1 = v[37]; const float i2 = v[38]; const float i3 = v[39]; const float i4 = v[40]; const float i5 = v[41]; const float i6 = v[42]; const float i7 = v[43]; const float i8 = v[44]; const float i9 = v[45]; const float i10 = v[46]; const float i11 = v[47]; const float i12 = v[48];
      v[36] = fmaf(24.75f, i5, fmaf(6.875f, i3, 0.375f * i1));
      v[37] = fmaf(5.15625f, i4, fmaf(1.375f, i2, 0.03125f * i0));
      v[38] = fmaf(-1.5f, i5, fmaf(1.25f, i3, 0.25f * i1));
      v[39] = fmaf(-0.84375f, i4, fmaf(0.375f, i2, 0.03125f * i0));
      v[40] = fmaf(0.25f, i5, fmaf(-0.375f, i3, 0.125f * i1));
      v[41] = fmaf(0.15625f, i4, fmaf(-0.125f, i2, 0.03125f * i0));
      v[42] = fmaf(0.015625f, i12, fmaf(-0.09375f, i10, fmaf(0.234375f, i8, -0.3125f * i6)));
      v[43] = fmaf(0.0625f, i11, fmaf(-0.3125f, i9, 0.625f * i7));
      v[44] = fmaf(0.03125f, i12, fmaf(0.0625f, i10, fmaf(-0.53125f, i8, 0.875f * i6)));
      v[45] = fmaf(0.1875f, i11, fmaf(0.0625f, i9, -1.125f * i7));
      v[46] = fmaf(0.03125f, i12, fmaf(0.8125f, i10, fmaf(0.46875f, i8, -2.625f * i6)));
      v[47] = fmaf(0.3125f, i11, fmaf(3.4375f, i9, 4.125f * i7));
      v[48] = fmaf(0.03125f, i12, fmaf(2.0625f, i10, fmaf(15.46875f, i8, 28.875f * i6)));
    }
    {
      const float i0 = v[49]; const float i1 = v[50]; const float i2 = v[51]; const float i3 = v[52]; const float i4 = v[53]; const float i5 = v[54]; const float i6 = v[55]; const float i7 = v[56]; const float i8 = v[57]; const float i9 = v[58]; const float i10 = v[59]; const float i11 = v[60]; const float i12 = v[61]; const float i13 = v[62]; const float i14 = v[63];
      v[49] = fmaf(46.921875f, i6, fmaf(15.640625f, i4, fmaf(1.421875f, i2, 0.015625f * i0)));
      v[50] = fmaf(8.9375f, i5, fmaf(3.25f, i3, 0.1875f * i1));
      v[51] = fmaf(-2.578125f, i6, fmaf(1.890625f, i4, fmaf(0.671875f, i2, 0.015625f * i0)));
      v[52] = fmaf(-1.375f, i5, fmaf(0.5f, i3, 0.125f * i1));
      v[53] = fmaf(0.421875f, i6, fmaf(-0.609375f, i4, fmaf(0.171875f, i2, 0.015625f * i0)));
      v[54] = fmaf(0.3125f, i5, fmaf(-0.25f, i3, 0.0625f * i1));
      v[55] = fmaf(-0.078125f, i6, fmaf(0.140625f, i4, fmaf(-0.078125f, i2, 0.015625f * i0)));
      v[56] = fmaf(0.0078125f, i14, fmaf(-0.0546875f, i12, fmaf(0.1640625f, i10, -0.2734375f * i8)));
      v[57] = fmaf(0.03125f, i13, fmaf(-0.1875f, i11, fmaf(0.46875f, i9, -0.625f * i7)));
      v[58] = fmaf(0.015625f, i14, fmaf(0.015625f, i12, fmaf(-0.296875f, i10, 0.703125f * i8)));
      v[59] = fmaf(0.09375f, i13, fmaf(-0.0625f, i11, fmaf(-0.59375f, i9, 1.125f * i7)));
      v[60] = fmaf(0.015625f, i14, fmaf(0.390625f, i12, fmaf(-0.171875f, i10, -1.546875f * i8)));
      v[61] = fmaf(0.15625f, i13, fmaf(1.5625f, i11, fmaf(0.34375f, i9, -4.125f * i7)));
      v[62] = fmaf(0.015625f, i14, fmaf(1.015625f, i12, fmaf(6.703125f, i10, 6.703125f * i8)));
      v[63] = fmaf(0.21875f, i13, fmaf(5.6875f, i11, fmaf(31.28125f, i9, 53.625f * i7)));
    }
  }
};
template <> struct BApply<8, false> {
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[1]; const float i1 = v[2]; const float i2 = v[3];
      v[1] = 1.0f * i0;
      v[2] = 2.0f * i2;
      v[3] = 0.5f * i1;
    }
    {
      const float i0 = v[4]; const float i1 = v[5]; const float i2 = v[6]; const float i3 = v[7]; const float i4 = v[8];
      v[4] = 0.5f * i1;
      v[5] = 2.0f * i0;
      v[6] = fmaf(3.0f, i4, -0.5f * i2);
      v[7] = 1.0f * i3;
      v[8] = fmaf(0.5f, i4, 0.25f * i2);
    }
    {
      const float i0 = v[9]; const float i1 = v[10]; const float i2 = v[11]; const float i3 = v[12]; const float i4 = v[13]; const float i5 = v[14]; const float i6 = v[15];
      v[9] = fmaf(0.25f, i2, 0.25f * i0);
      v[10] = 1.0f * i1;
      v[11] = fmaf(-0.25f, i2, 3.75f * i0);
      v[12] = fmaf(5.0f, i6, -1.0f * i4);
      v[13] = fmaf(1.25f, i5, -0.375f * i3);
      v[14] = fmaf(1.5f, i6, 0.5f * i4);
      v[15] = fmaf(0.25f, i5, 0.125f * i3);
    }
    {
      const float i0 = v[16]; const float i1 = v[17]; const float i2 = v[18]; const float i3 = v[19]; const float i4 = v[20]; const float i5 = v[21]; const float i6 = v[22]; const float i7 = v[23]; const float i8 = v[24];
      v[16] = fmaf(0.125f, i3, 0.125f * i1);
      v[17] = fmaf(0.5f, i2, 1.0f * i0);
      v[18] = fmaf(-0.25f, i3, 1.75f * i1);
      v[19] = fmaf(-0.5f, i2, 7.0f * i0);
      v[20] = fmaf(8.75f, i8, fmaf(-1.25f, i6, 0.375f * i4));
      v[21] = fmaf(1.75f, i7, -0.75f * i5);
      v[22] = fmaf(3.5f, i8, fmaf(0.5f, i6, -0.25f * i4));
      v[23] = fmaf(0.75f, i7, 0.25f * i5);
      v[24] = fmaf(0.125f, i8, fmaf(0.125f, i6, 0.0625f * i4));
    }
    {
      const float i0 = v[25]; const float i1 = v[26]; const float i2 = v[27]; const float i3 = v[28]; const float i4 = v[29]; const float i5 = v[30]; const float i6 = v[31]; const float i7 = v[32]; const float i8 = v[33]; const float i9 = v[34]; const float i10 = v[35];
      v[25] = fmaf(0.0625f, i4, fmaf(0.0625f, i2, 0.0625f * i0));
      v[26] = fmaf(0.25f, i3, 0.5f * i1);
      v[27] = fmaf(-0.1875f, i4, fmaf(0.8125f, i2, 2.8125f * i0));
      v[28] = fmaf(-0.5f, i3, 3.0f * i1);
      v[29] = fmaf(0.125f, i4, fmaf(-0.875f, i2, 13.125f * i0));
      v[30] = fmaf(15.75f, i10, fmaf(-1.75f, i8, 0.75f * i6));
      v[31] = fmaf(2.625f, i9, fmaf(-0.875f, i7, 0.3125f * i5));
      v[32] = fmaf(7.5f, i10, fmaf(0.5f, i8, -0.5f * i6));
      v[33] = fmaf(1.6875f, i9, fmaf(0.1875f, i7, -0.15625f * i5));
      v[34] = fmaf(0.625f, i10, fmaf(0.375f, i8, 0.125f * i6));
      v[35] = fmaf(0.0625f, i9, fmaf(0.0625f, i7, 0.03125f * i5));
    }
    {
      const float i0 = v[36]; const float i1 = v[37]; const float i2 = v[38]; const float i3 = v[39]; const float i4 = v[40]; const float i5 = v[41]; const float i6 = v[42]; const float i7 = v[43]; const float i8 = v[44]; const float i9 = v[45]; const float i10 = v[46]; const float i11 = v[47]; const float i12 = v[48];
      v[36] = fmaf(0.03125f, i5, fmaf(0.03125f, i3, 0.03125f * i1));
      v[37] = fmaf(0.125f, i4, fmaf(0.25f, i2, 0.375f * i0));
      v[38] = fmaf(-0.125f, i5, fmaf(0.375f, i3, 1.375f * i1));
      v[39] = fmaf(-0.375f, i4, fmaf(1.25f, i2, 6.875f * i0));
      v[40] = fmaf(0.15625f, i5, fmaf(-0.84375f, i3, 5.15625f * i1));
      v[41] = fmaf(0.25f, i4, fmaf(-1.5f, i2, 24.75f * i0));
      v[42] = fmaf(28.875f, i12, fmaf(-2.625f, i10, fmaf(0.875f, i8, -0.3125f * i6)));
      v[43] = fmaf(4.125f, i11, fmaf(-1.125f, i9, 0.625f * i7));
      v[44] = fmaf(15.46875f, i12, fmaf(0.46875f, i10, fmaf(-0.53125f, i8, 0.234375f * i6)));
      v[45] = fmaf(3.4375f, i11, fmaf(0.0625f, i9, -0.3125f * i7));
      v[46] = fmaf(2.0625f, i12, fmaf(0.8125f, i10, fmaf(0.0625f, i8, -0.09375f * i6)));
      v[47] = fmaf(0.3125f, i11, fmaf(0.1875f, i9, 0.0625f * i7));
      v[48] = fmaf(0.03125f, i12, fmaf(0.03125f, i10, fmaf(0.03125f, i8, 0.015625f * i6)));
    }
    {
      const float i0 = v[49]; const float i1 = v[50]; const float i2 = v[51]; const float i3 = v[52]; const float i4 = v[53]; const float i5 = v[54]; const float i6 = v[55]; const float i7 = v[56]; const float i8 = v[57]; const float i9 = v[58]; const float i10 = v[59]; const float i11 = v[60]; const float i12 = v[61]; const float i13 = v[62]; const float i14 = v[63];
      v[49] = fmaf(0.015625f, i6, fmaf(0.015625f, i4, fmaf(0.015625f, i2, 0.015625f * i0)));
      v[50] = fmaf(0.0625f, i5, fmaf(0.125f, i3, 0.1875f * i1));
      v[51] = fmaf(-0.078125f, i6, fmaf(0.171875f, i4, fmaf(0.671875f, i2, 1.421875f * i0)));
      v[52] = fmaf(-0.25f, i5, fmaf(0.5f, i3, 3.25f * i1));
      v[53] = fmaf(0.140625f, i6, fmaf(-0.609375f, i4, fmaf(1.890625f, i2, 15.640625f * i0)));
      v[54] = fmaf(0.3125f, i5, fmaf(-1.375f, i3, 8.9375f * i1));
      v[55] = fmaf(-0.078125f, i6, fmaf(0.421875f, i4, fmaf(-2.578125f, i2, 46.921875f * i0)));
      v[56] = fmaf(53.625f, i14, fmaf(-4.125f, i12, fmaf(1.125f, i10, -0.625f * i8)));
      v[57] = fmaf(6.703125f, i13, fmaf(-1.546875f, i11, fmaf(0.703125f, i9, -0.2734375f * i7)));
      v[58] = fmaf(31.28125f, i14, fmaf(0.34375f, i12, fmaf(-0.59375f, i10, 0.46875f * i8)));
      v[59] = fmaf(6.703125f, i13, fmaf(-0.171875f, i11, fmaf(-0.296875f, i9, 0.1640625f * i7)));
      v[60] = fmaf(5.6875f, i14, fmaf(1.5625f, i12, fmaf(-0.0625f, i10, -0.1875f * i8)));
      v[61] = fmaf(1.015625f, i13, fmaf(0.390625f, i11, fmaf(0.015625f, i9, -0.0546875f * i7)));
      v[62] = fmaf(0.21875f, i14, fmaf(0.15625f, i12, fmaf(0.09375f, i10, 0.03125f * i8)));
      v[63] = fmaf(0.015625f, i13, fmaf(0.015625f, i11, fmaf(0.015625f, i9, 0.0078125f * i7)));
    }
    {
      const float i0 = v[64]; const float i1 = v[65]; const float i2 = v[66]; const float i3 = v[67]; const float i4 = v[68]; const float i5 = v[69]; const float i6 = v[70]; const float i7 = v[71]; const float i8 = v[72]; const float i9 = v[73]; const float i10 = v[74]; const float i11 = v[75]; const float i12 = v[76]; const float i13 = v[77]; const float i14 = v[78]; const float i15 = v[79]; const float i16 = v[80];
      v[64] = fmaf(0.0078125f, i7, fmaf(0.0078125f, i5, fmaf(0.0078125f, i3, 0.0078125f * i1)));
      v[65] = fmaf(0.03125f, i6, fmaf(0.0625f, i4, fmaf(0.09375f, i2, 0.125f * i0)));
      v[66] = fmaf(-0.046875f, i7, fmaf(0.078125f, i5, fmaf(0.328125f, i3, 0.703125f * i1)));
      v[67] = fmaf(-0.15625f, i6, fmaf(0.1875f, i4, fmaf(1.53125f, i2, 4.375f * i0)));
      v[68] = fmaf(0.109375f, i7, fmaf(-0.390625f, i5, fmaf(0.609375f, i3, 7.109375f * i1)));
      v[69] = fmaf(0.28125f, i6, fmaf(-0.9375f, i4, fmaf(2.84375f, i2, 34.125f * i0)));
      v[70] = fmaf(-0.109375f, i7, fmaf(0.515625f, i5, fmaf(-2.234375f, i3, 15.640625f * i1)));
      v[71] = fmaf(-0.15625f, i6, fmaf(0.6875f, i4, fmaf(-4.46875f, i2, 89.375f * i0)));
      v[72] = fmaf(100.546875f, i16, fmaf(-6.703125f, i14, fmaf(1.546875f, i12, fmaf(-0.703125f, i10, 0.2734375f * i8))));
      v[73] = fmaf(11.171875f, i15, fmaf(-2.234375f, i13, fmaf(0.859375f, i11, -0.546875f * i9)));
      v[74] = fmaf(62.5625f, i16, fmaf(-0.6875f, i12, fmaf(0.5f, i10, -0.21875f * i8)));
      v[75] = fmaf(12.796875f, i15, fmaf(-0.609375f, i13, fmaf(-0.265625f, i11, 0.328125f * i9)));
      v[76] = fmaf(14.21875f, i16, fmaf(2.84375f, i14, fmaf(-0.28125f, i12, fmaf(-0.15625f, i10, 0.109375f * i8))));
      v[77] = fmaf(2.734375f, i15, fmaf(0.703125f, i13, fmaf(-0.078125f, i11, -0.109375f * i9)));
      v[78] = fmaf(0.9375f, i16, fmaf(0.5f, i14, fmaf(0.1875f, i12, -0.03125f * i8)));
      v[79] = fmaf(0.109375f, i15, fmaf(0.078125f, i13, fmaf(0.046875f, i11, 0.015625f * i9)));
      v[80] = fmaf(0.0078125f, i16, fmaf(0.0078125f, i14, fmaf(0.0078125f, i12, fmaf(0.0078125f, i10, 0.00390625f * i8))));
    }
  }
};
template <> struct BApply<8, true> {
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[1]; const float i1 = v[2]; const float i2 = v[3];
      v[1] = 1.0f * i0;
      v[2] = 0.5f * i2;
      v[3] = 2.0f * i1;
    }
    {
      const float i0 = v[4]; const float i1 = v[5]; const float i2 = v[6]; const float i3 = v[7]; const float i4 = v[8];
      v[4] = 2.0f * i1;
      v[5] = 0.5f * i0;
      v[6] = fmaf(0.25f, i4, -0.5f * i2);
      v[7] = 1.0f * i3;
      v[8] = fmaf(0.5f, i4, 3.0f * i2);
    }
    {
      const float i0 = v[9]; const float i1 = v[10]; const float i2 = v[11]; const float i3 = v[12]; const float i4 = v[13]; const float i5 = v[14]; const float i6 = v[15];
      v[9] = fmaf(3.75f, i2, 0.25f * i0);
      v[10] = 1.0f * i1;
      v[11] = fmaf(-0.25f, i2, 0.25f * i0);
      v[12] = fmaf(0.125f, i6, -0.375f * i4);
      v[13] = fmaf(0.5f, i5, -1.0f * i3);
      v[14] = fmaf(0.25f, i6, 1.25f * i4);
      v[15] = fmaf(1.5f, i5, 5.0f * i3);
    }
    {
      const float i0 = v[16]; const float i1 = v[17]; const float i2 = v[18]; const float i3 = v[19]; const float i4 = v[20]; const float i5 = v[21]; const float i6 = v[22]; const float i7 = v[23]; const float i8 = v[24];
      v[16] = fmaf(7.0f, i3, 1.0f * i1);
      v[17] = fmaf(1.75f, i2, 0.125f * i0);
      v[18] = fmaf(-0.5f, i3, 0.5f * i1);
      v[19] = fmaf(-0.25f, i2, 0.125f * i0);
      v[20] = fmaf(0.0625f, i8, fmaf(-0.25f, i6, 0.375f * i4));
      v[21] = fmaf(0.25f, i7, -0.75f * i5);
      v[22] = fmaf(0.125f, i8, fmaf(0.5f, i6, -1.25f * i4));
      v[23] = fmaf(0.75f, i7, 1.75f * i5);
      v[24] = fmaf(0.125f, i8, fmaf(3.5f, i6, 8.75f * i4));
    }
    {
      const float i0 = v[25]; const float i1 = v[26]; const float i2 = v[27]; const float i3 = v[28]; const float i4 = v[29]; const float i5 = v[30]; const float i6 = v[31]; const float i7 = v[32]; const float i8 = v[33]; const float i9 = v[34]; const float i10 = v[35];
      v[25] = fmaf(13.125f, i4, fmaf(2.8125f, i2, 0.0625f * i0));
      v[26] = fmaf(3.0f, i3, 0.5f * i1);
      v[27] = fmaf(-0.875f, i4, fmaf(0.8125f, i2, 0.0625f * i0));
      v[28] = fmaf(-0.5f, i3, 0.25f * i1);
      v[29] = fmaf(0.125f, i4, fmaf(-0.1875f, i2, 0.0625f * i0));
      v[30] = fmaf(0.03125f, i10, fmaf(-0.15625f, i8, 0.3125f * i6));
      v[31] = fmaf(0.125f, i9, fmaf(-0.5f, i7, 0.75f * i5));
      v[32] = fmaf(0.0625f, i10, fmaf(0.1875f, i8, -0.875f * i6));
      v[33] = fmaf(0.375f, i9, fmaf(0.5f, i7, -1.75f * i5));
      v[34] = fmaf(0.0625f, i10, fmaf(1.6875f, i8, 2.625f * i6));
      v[35] = fmaf(0.625f, i9, fmaf(7.5f, i7, 15.75f * i5));
    }
    {
      const float i0 = v[36]; const float i1 = v[37]; const float i2 = v[38]; const float i3 = v[39]; const float i4 = v[40]; const float i5 = v[41]; const float i6 = v[42]; const float i7 = v[43]; const float i8 = v[44]; const float i9 = v[45]; const float i10 = v[46]; const float i11 = v[47]; const float i12 = v[48];
      v[36] = fmaf(24.75f, i5, fmaf(6.875f, i3, 0.375f * i1));
      v[37] = fmaf(5.15625f, i4, fmaf(1.375f, i2, 0.03125f * i0));
      v[38] = fmaf(-1.5f, i5, fmaf(1.25f, i3, 0.25f * i1));
      v[39] = fmaf(-0.84375f, i4, fmaf(0.375f, i2, 0.03125f * i0));
      v[40] = fmaf(0.25f, i5, fmaf(-0.375f, i3, 0.125f * i1));
      v[41] = fmaf(0.15625f, i4, fmaf(-0.125f, i2, 0.03125f * i0));
      v[42] = fmaf(0.015625f, i12, fmaf(-0.09375f, i10, fmaf(0.234375f, i8, -0.3125f * i6)));
      v[43] = fmaf(0.0625f, i11, fmaf(-0.3125f, i9, 0.625f * i7));
      v[44] = fmaf(0.03125f, i12, fmaf(0.0625f, i10, fmaf(-0.53125f, i8, 0.875f * i6)));
      v[45] = fmaf(0.1875f, i11, fmaf(0.0625f, i9, -1.125f * i7));
      v[46] = fmaf(0.03125f, i12, fmaf(0.8125f, i10, fmaf(0.46875f, i8, -2.625f * i6)));
      v[47] = fmaf(0.3125f, i11, fmaf(3.4375f, i9, 4.125f * i7));
      v[48] = fmaf(0.03125f, i12, fmaf(2.0625f, i10, fmaf(15.46875f, i8, 28.875f * i6)));
    }
    {
      const float i0 = v[49]; const float i1 = v[50]; const float i2 = v[51]; const float i3 = v[52]; const float i4 = v[53]; const float i5 = v[54]; const float i6 = v[55]; const float i7 = v[56]; const float i8 = v[57]; const float i9 = v[58]; const float i10 = v[59]; const float i11 = v[60]; const float i12 = v[61]; const float i13 = v[62]; const float i14 = v[63];
      v[49] = fmaf(46.921875f, i6, fmaf(15.640625f, i4, fmaf(1.421875f, i2, 0.015625f * i0)));
      v[50] = fmaf(8.9375f, i5, fmaf(3.25f, i3, 0.1875f * i1));
      v[51] = fmaf(-2.578125f, i6, fmaf(1.890625f, i4, fmaf(0.671875f, i2, 0.015625f * i0)));
      v[52] = fmaf(-1.375f, i5, fmaf(0.5f, i3, 0.125f * i1));
      v[53] = fmaf(0.421875f, i6, fmaf(-0.609375f, i4, fmaf(0.171875f, i2, 0.015625f * i0)));
      v[54] = fmaf(0.3125f, i5, fmaf(-0.25f, i3, 0.0625f * i1));
      v[55] = fmaf(-0.078125f, i6, fmaf(0.140625f, i4, fmaf(-0.078125f, i2, 0.015625f * i0)));
      v[56] = fmaf(0.0078125f, i14, fmaf(-0.0546875f, i12, fmaf(0.1640625f, i10, -0.2734375f * i8)));
      v[57] = fmaf(0.03125f, i13, fmaf(-0.1875f, i11, fmaf(0.46875f, i9, -0.625f * i7)));
      v[58] = fmaf(0.015625f, i14, fmaf(0.015625f, i12, fmaf(-0.296875f, i10, 0.703125f * i8)));
      v[59] = fmaf(0.09375f, i13, fmaf(-0.0625f, i11, fmaf(-0.59375f, i9, 1.125f * i7)));
      v[60] = fmaf(0.015625f, i14, fmaf(0.390625f, i12, fmaf(-0.171875f, i10, -1.546875f * i8)));
      v[61] = fmaf(0.15625f, i13, fmaf(1.5625f, i11, fmaf(0.34375f, i9, -4.125f * i7)));
      v[62] = fmaf(0.015625f, i14, fmaf(1.015625f, i12, fmaf(6.703125f, i10, 6.703125f * i8)));
      v[63] = fmaf(0.21875f, i13, fmaf(5.6875f, i11, fmaf(31.28125f, i9, 53.625f * i7)));
    }
    {
      const float i0 = v[64]; const float i1 = v[65]; const float i2 = v[66]; const float i3 = v[67]; const float i4 = v[68]; const float i5 = v[69]; const float i6 = v[70]; const float i7 = v[71]; const float i8 = v[72]; const float i9 = v[73]; const float i10 = v[74]; const float i11 = v[75]; const float i12 = v[76]; const float i13 = v[77]; const float i14 = v[78]; const float i15 = v[79]; const float i16 = v[80];
      v[64] = fmaf(89.375f, i7, fmaf(34.125f, i5, fmaf(4.375f, i3, 0.125f * i1)));
      v[65] = fmaf(15.640625f, i6, fmaf(7.109375f, i4, fmaf(0.703125f, i2, 0.0078125f * i0)));
      v[66] = fmaf(-4.46875f, i7, fmaf(2.84375f, i5, fmaf(1.53125f, i3, 0.09375f * i1)));
      v[67] = fmaf(-2.234375f, i6, fmaf(0.609375f, i4, fmaf(0.328125f, i2, 0.0078125f * i0)));
      v[68] = fmaf(0.6875f, i7, fmaf(-0.9375f, i5, fmaf(0.1875f, i3, 0.0625f * i1)));
      v[69] = fmaf(0.515625f, i6, fmaf(-0.390625f, i4, fmaf(0.078125f, i2, 0.0078125f * i0)));
      v[70] = fmaf(-0.15625f, i7, fmaf(0.28125f, i5, fmaf(-0.15625f, i3, 0.03125f * i1)));
      v[71] = fmaf(-0.109375f, i6, fmaf(0.109375f, i4, fmaf(-0.046875f, i2, 0.0078125f * i0)));
      v[72] = fmaf(0.00390625f, i16, fmaf(-0.03125f, i14, fmaf(0.109375f, i12, fmaf(-0.21875f, i10, 0.2734375f * i8))));
      v[73] = fmaf(0.015625f, i15, fmaf(-0.109375f, i13, fmaf(0.328125f, i11, -0.546875f * i9)));
      v[74] = fmaf(0.0078125f, i16, fmaf(-0.15625f, i12, fmaf(0.5f, i10, -0.703125f * i8)));
      v[75] = fmaf(0.046875f, i15, fmaf(-0.078125f, i13, fmaf(-0.265625f, i11, 0.859375f * i9)));
      v[76] = fmaf(0.0078125f, i16, fmaf(0.1875f, i14, fmaf(-0.28125f, i12, fmaf(-0.6875f, i10, 1.546875f * i8))));
      v[77] = fmaf(0.078125f, i15, fmaf(0.703125f, i13, fmaf(-0.609375f, i11, -2.234375f * i9)));
      v[78] = fmaf(0.0078125f, i16, fmaf(0.5f, i14, fmaf(2.84375f, i12, -6.703125f * i8)));
      v[79] = fmaf(0.109375f, i15, fmaf(2.734375f, i13, fmaf(12.796875f, i11, 11.171875f * i9)));
      v[80] = fmaf(0.0078125f, i16, fmaf(0.9375f, i14, fmaf(14.21875f, i12, fmaf(62.5625f, i10, 100.546875f * i8))));
    }
  }
};
template <> struct BApply<9, false> {
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[1]; const float i1 = v[2]; const float i2 = v[3];
      v[1] = 1.0f * i0;
      v[2] = 2.0f * i2;
      v[3] = 0.5f * i1;
    }
    {
      const float i0 = v[4]; const float i1 = v[5]; const float i2 = v[6]; const float i3 = v[7]; const float i4 = v[8];
      v[4] = 0.5f * i1;
      v[5] = 2.0f * i0;
      v[6] = fmaf(3.0f, i4, -0.5f * i2);
      v[7] = 1.0f * i3;
      v[8] = fmaf(0.5f, i4, 0.25f * i2);
    }
    {
      const float i0 = v[9]; const float i1 = v[10]; const float i2 = v[11]; const float i3 = v[12]; const float i4 = v[13]; const float i5 = v[14]; const float i6 = v[15];
      v[9] = fmaf(0.25f, i2, 0.25f * i0);
      v[10] = 1.0f * i1;
      v[11] = fmaf(-0.25f, i2, 3.75f * i0);
      v[12] = fmaf(5.0f, i6, -1.0f * i4);
      v[13] = fmaf(1.25f, i5, -0.375f * i3);
      v[14] = fmaf(1.5f, i6, 0.5f * i4);
      v[15] = fmaf(0.25f, i5, 0.125f * i3);
    }
    {
      const float i0 = v[16]; const float i1 = v[17]; const float i2 = v[18]; const float i3 = v[19]; const float i4 = v[20]; const float i5 = v[21]; const float i6 = v[22]; const float i7 = v[23]; const float i8 = v[24];
      v[16] = fmaf(0.125f, i3, 0.125f * i1);
      v[17] = fmaf(0.5f, i2, 1.0f * i0);
      v[18] = fmaf(-0.25f, i3, 1.75f * i1);
      v[19] = fmaf(-0.5f, i2, 7.0f * i0);
      v[20] = fmaf(8.75f, i8, fmaf(-1.25f, i6, 0.375f * i4));
      v[21] = fmaf(1.75f, i7, -0.75f * i5);
      v[22] = fmaf(3.5f, i8, fmaf(0.5f, i6, -0.25f * i4));
      v[23] = fmaf(0.75f, i7, 0.25f * i5);
      v[24] = fmaf(0.125f, i8, fmaf(0.125f, i6, 0.0625f * i4));
    }
    {
      const float i0 = v[25]; const float i1 = v[26]; const float i2 = v[27]; const float i3 = v[28]; const float i4 = v[29]; const float i5 = v[30]; const float i6 = v[31]; const float i7 = v[32]; const float i8 = v[33]; const float i9 = v[34]; const float i10 = v[35];
      v[25] = fmaf(0.0625f, i4, fmaf(0.0625f, i2, 0.0625f * i0));
      v[26] = fmaf(0.25f, i3, 0.5f * i1);
      v[27] = fmaf(-0.1875f, i4, fmaf(0.8125f, i2, 2.8125f * i0));
      v[28] = fmaf(-0.5f, i3, 3.0f * i1);
      v[29] = fmaf(0.125f, i4, fmaf(-0.875f, i2, 13.125f * i0));
      v[30] = fmaf(15.75f, i10, fmaf(-1.75f, i8, 0.75f * i6));
      v[31] = fmaf(2.625f, i9, fmaf(-0.875f, i7, 0.3125f * i5));
      v[32] = fmaf(7.5f, i10, fmaf(0.5f, i8, -0.5f * i6));
      v[33] = fmaf(1.6875f, i9, fmaf(0.1875f, i7, -0.15625f * i5));
      v[34] = fmaf(0.625f, i10, fmaf(0.375f, i8, 0.125f * i6));
      v[35] = fmaf(0.0625f, i9, fmaf(0.0625f, i7, 0.03125f * i5));
    }
    {
      const float i0 = v[36]; const float i1 = v[37]; const float i2 = v[38]; const float i3 = v[39]; const float i4 = v[40]; const float i5 = v[41]; const float i6 = v[42]; const float i7 = v[43]; const float i8 = v[44]; const float i9 = v[45]; const float i10 = v[46]; const float i11 = v[47]; const float i12 = v[48];
      v[36] = fmaf(0.03125f, i5, fmaf(0.03125f, i3, 0.03125f * i1));
      v[37] = fmaf(0.125f, i4, fmaf(0.25f, i2, 0.375f * i0));
      v[38] = fmaf(-0.125f, i5, fmaf(0.375f, i3, 1.375f * i1));
      v[39] = fmaf(-0.375f, i4, fmaf(1.25f, i2, 6.875f * i0));
      v[40] = fmaf(0.15625f, i5, fmaf(-0.84375f, i3, 5.15625f * i1));
      v[41] = fmaf(0.25f, i4, fmaf(-1.5f, i2, 24.75f * i0));
      v[42] = fmaf(28.875f, i12, fmaf(-2.625f, i10, fmaf(0.875f, i8, -0.3125f * i6)));
      v[43] = fmaf(4.125f, i11, fmaf(-1.125f, i9, 0.625f * i7));
      v[44] = fmaf(15.46875f, i12, fmaf(0.46875f, i10, fmaf(-0.53125f, i8, 0.234375f * i6)));
      v[45] = fmaf(3.4375f, i11, fmaf(0.0625f, i9, -0.3125f * i7));
      v[46] = fmaf(2.0625f, i12, fmaf(0.8125f, i10, fmaf(0.0625f, i8, -0.09375f * i6)));
      v[47] = fmaf(0.3125f, i11, fmaf(0.1875f, i9, 0.0625f * i7));
      v[48] = fmaf(0.03125f, i12, fmaf(0.03125f, i10, fmaf(0.03125f, i8, 0.015625f * i6)));
    }
    {
      const float i0 = v[49]; const float i1 = v[50]; const float i2 = v[51]; const float i3 = v[52]; const float i4 = v[53]; const float i5 = v[54]; const float i6 = v[55]; const float i7 = v[56]; const float i8 = v[57]; const float i9 = v[58]; const float i10 = v[59]; const float i11 = v[60]; const float i12 = v[61]; const float i13 = v[62]; const float i14 = v[63];
      v[49] = fmaf(0.015625f, i6, fmaf(0.015625f, i4, fmaf(0.015625f, i2, 0.015625f * i0)));
      v[50] = fmaf(0.0625f, i5, fmaf(0.125f, i3, 0.1875f * i1));
      v[51] = fmaf(-0.078125f, i6, fmaf(0.171875f, i4, fmaf(0.671875f, i2, 1.421875f * i0)));
      v[52] = fmaf(-0.25f, i5, fmaf(0.5f, i3, 3.25f * i1));
      v[53] = fmaf(0.140625f, i6, fmaf(-0.609375f, i4, fmaf(1.890625f, i2, 15.640625f * i0)));
      v[54] = fmaf(0.3125f, i5, fmaf(-1.375f, i3, 8.9375f * i1));
      v[55] = fmaf(-0.078125f, i6, fmaf(0.421875f, i4, fmaf(-2.578125f, i2, 46.921875f * i0)));
      v[56] = fmaf(53.625f, i14, fmaf(-4.125f, i12, fmaf(1.125f, i10, -0.625f * i8)));
      v[57] = fmaf(6.703125f, i13, fmaf(-1.546875f, i11, fmaf(0.703125f, i9, -0.2734375f * i7)));
      v[58] = fmaf(31.28125f, i14, fmaf(0.34375f, i12, fmaf(-0.59375f, i10, 0.46875f * i8)));
      v[59] = fmaf(6.703125f, i13, fmaf(-0.171875f, i11, fmaf(-0.296875f, i9, 0.1640625f * i7)));
      v[60] = fmaf(5.6875f, i14, fmaf(1.5625f, i12, fmaf(-0.0625f, i10, -0.1875f * i8)));
      v[61] = fmaf(1.015625f, i13, fmaf(0.390625f, i11, fmaf(0.015625f, i9, -0.0546875f * i7)));
      v[62] = fmaf(0.21875f, i14, fmaf(0.15625f, i12, fmaf(0.09375f, i10, 0.03125f * i8)));
      v[63] = fmaf(0.015625f, i13, fmaf(0.015625f, i11, fmaf(0.015625f, i9, 0.0078125f * i7)));
    }
    {
      const float i0 = v[64]; const float i1 = v[65]; const float i2 = v[66]; const float i3 = v[67]; const float i4 = v[68]; const float i5 = v[69]; const float i6 = v[70]; const float i7 = v[71]; const float i8 = v[72]; const float i9 = v[73]; const float i10 = v[74]; const float i11 = v[75]; const float i12 = v[76]; const float i13 = v[77]; const float i14 = v[78]; const float i15 = v[79]; const float i16 = v[80];
      v[64] = fmaf(0.0078125f, i7, fmaf(0.0078125f, i5, fmaf(0.0078125f, i3, 0.0078125f * i1)));
      v[65] = fmaf(0.03125f, i6, fmaf(0.0625f, i4, fmaf(0.09375f, i2, 0.125f * i0)));
      v[66] = fmaf(-0.046875f, i7, fmaf(0.078125f, i5, fmaf(0.328125f, i3, 0.703125f * i1)));
      v[67] = fmaf(-0.15625f, i6, fmaf(0.1875f, i4, fmaf(1.53125f, i2, 4.375f * i0)));
      v[68] = fmaf(0.109375f, i7, fmaf(-0.390625f, i5, fmaf(0.609375f, i3, 7.109375f * i1)));
      v[69] = fmaf(0.28125f, i6, fmaf(-0.9375f, i4, fmaf(2.84375f, i2, 34.125f * i0)));
      v[70] = fmaf(-0.109375f, i7, fmaf(0.515625f, i5, fmaf(-2.234375f, i3, 15.640625f * i1)));
      v[71] = fmaf(-0.15625f, i6, fmaf(0.6875f, i4, fmaf(-4.46875f, i2, 89.375f * i0)));
      v[72] = fmaf(100.546875f, i16, fmaf(-6.703125f, i14, fmaf(1.546875f, i12, fmaf(-0.703125f, i10, 0.2734375f * i8))));
      v[73] = fmaf(11.171875f, i15, fmaf(-2.234375f, i13, fmaf(0.859375f, i11, -0.546875f * i9)));
      v[74] = fmaf(62.5625f, i16, fmaf(-0.6875f, i12, fmaf(0.5f, i10, -0.21875f * i8)));
      v[75] = fmaf(12.796875f, i15, fmaf(-0.609375f, i13, fmaf(-0.265625f, i11, 0.328125f * i9)));
      v[76] = fmaf(14.21875f, i16, fmaf(2.84375f, i14, fmaf(-0.28125f, i12, fmaf(-0.15625f, i10, 0.109375f * i8))));
      v[77] = fmaf(2.734375f, i15, fmaf(0.703125f, i13, fmaf(-0.078125f, i11, -0.109375f * i9)));
      v[78] = fmaf(0.9375f, i16, fmaf(0.5f, i14, fmaf(0.1875f, i12, -0.03125f * i8)));
      v[79] = fmaf(0.109375f, i15, fmaf(0.078125f, i13, fmaf(0.046875f, i11, 0.015625f * i9)));
      v[80] = fmaf(0.0078125f, i16, fmaf(0.0078125f, i14, fmaf(0.0078125f, i12, fmaf(0.0078125f, i10, 0.00390625f * i8))));
    }
    {
      const float i0 = v[81]; const float i1 = v[82]; const float i2 = v[83]; const float i3 = v[84]; const float i4 = v[85]; const float i5 = v[86]; const float i6 = v[87]; const float i7 = v[88]; const float i8 = v[89]; const float i9 = v[90]; const float i10 = v[91]; const float i11 = v[92]; const float i12 = v[93]; const float i13 = v[94]; const float i14 = v[95]; const float i15 = v[96]; const float i16 = v[97]; const float i17 = v[98]; const float i18 = v[99];
      v[81] = fmaf(0.00390625f, i8, fmaf(0.00390625f, i6, fmaf(0.00390625f, i4, fmaf(0.00390625f, i2, 0.00390625f * i0))));
      v[82] = fmaf(0.015625f, i7, fmaf(0.03125f, i5, fmaf(0.046875f, i3, 0.0625f * i1)));
      v[83] = fmaf(-0.02734375f, i8, fmaf(0.03515625f, i6, fmaf(0.16015625f, i4, fmaf(0.34765625f, i2, 0.59765625f * i0))));
      v[84] = fmaf(-0.09375f, i7, fmaf(0.0625f, i5, fmaf(0.71875f, i3, 2.125f * i1)));
      v[85] = fmaf(0.078125f, i8, fmaf(-0.234375f, i6, fmaf(0.140625f, i4, fmaf(3.203125f, i2, 11.953125f * i0))));
      v[86] = fmaf(0.21875f, i7, fmaf(-0.5625f, i5, fmaf(0.65625f, i3, 14.875f * i1)));
      v[87] = fmaf(-0.109375f, i8, fmaf(0.453125f, i6, fmaf(-1.421875f, i4, fmaf(4.265625f, i2, 72.515625f * i0))));
      v[88] = fmaf(-0.21875f, i7, fmaf(0.8125f, i5, fmaf(-3.65625f, i3, 27.625f * i1)));
      v[89] = fmaf(0.0546875f, i8, fmaf(-0.2578125f, i6, fmaf(1.1171875f, i4, fmaf(-7.8203125f, i2, 170.9296875f * i0))));
      v[90] = fmaf(189.921875f, i18, fmaf(-11.171875f, i16, fmaf(2.234375f, i14, fmaf(-0.859375f, i12, 0.546875f * i10))));
      v[91] = fmaf(18.9921875f, i17, fmaf(-3.3515625f, i15, fmaf(1.1171875f, i13, fmaf(-0.6015625f, i11, 0.24609375f * i9))));
      v[92] = fmaf(124.3125f, i18, fmaf(-0.8125f, i16, fmaf(-0.8125f, i14, fmaf(0.5625f, i12, -0.4375f * i10))));
      v[93] = fmaf(24.171875f, i17, fmaf(-1.421875f, i15, fmaf(-0.203125f, i13, fmaf(0.328125f, i11, -0.1640625f * i9))));
      v[94] = fmaf(33.46875f, i18, fmaf(5.03125f, i16, fmaf(-0.65625f, i14, fmaf(-0.09375f, i12, 0.21875f * i10))));
      v[95] = fmaf(6.640625f, i17, fmaf(1.171875f, i15, fmaf(-0.234375f, i13, fmaf(-0.078125f, i11, 0.0703125f * i9))));
      v[96] = fmaf(3.1875f, i18, fmaf(1.3125f, i16, fmaf(0.3125f, i14, fmaf(-0.0625f, i12, -0.0625f * i10))));
      v[97] = fmaf(0.46484375f, i17, fmaf(0.24609375f, i15, fmaf(0.08984375f, i13, fmaf(-0.00390625f, i11, -0.017578125f * i9))));
      v[98] = fmaf(0.0703125f, i18, fmaf(0.0546875f, i16, fmaf(0.0390625f, i14, fmaf(0.0234375f, i12, 0.0078125f * i10))));
      v[99] = fmaf(0.00390625f, i17, fmaf(0.00390625f, i15, fmaf(0.00390625f, i13, fmaf(0.00390625f, i11, 0.001953125f * i9))));
    }
  }
};
template <> struct BApply<9, true> {
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[1]; const float i1 = v[2]; const float i2 = v[3];
      v[1] = 1.0f * i0;
      v[2] = 0.5f * i2;
      v[3] = 2.0f * i1;
    }
    {
      const float i0 = v[4]; const float i1 = v[5]; const float i2 = v[6]; const float i3 = v[7]; const float i4 = v[8];
      v[4] = 2.0f * i1;
      v[5] = 0.5f * i0;
      v[6] = fmaf(0.25f, i4, -0.5f * i2);
      v[7] = 1.0f * i3;
      v[8] = fmaf(0.5f, i4, 3.0f * i2);
    }
    {
      const float i0 = v[9]; const float i1 = v[10]; const float i2 = v[11]; const float i3 = v[12]; const float i4 = v[13]; const float i5 = v[14]; const float i6 = v[15];
      v[9] = fmaf(3.75f, i2, 0.25f * i0);
      v[10] = 1.0f * i1;
      v[11] = fmaf(-0.25f, i2, 0.25f * i0);
      v[12] = fmaf(0.125f, i6, -0.375f * i4);
      v[13] = fmaf(0.5f, i5, -1.0f * i3);
      v[14] = fmaf(0.25f, i6, 1.25f * i4);
      v[15] = fmaf(1.5f, i5, 5.0f * i3);
    }
    {
      const float i0 = v[16]; const float i1 = v[17]; const float i2 = v[18]; const float i3 = v[19]; const float i4 = v[20]; const float i5 = v[21]; const float i6 = v[22]; const float i7 = v[23]; const float i8 = v[24];
      v[16] = fmaf(7.0f, i3, 1.0f * i1);
      v[17] = fmaf(1.75f, i2, 0.125f * i0);
      v[18] = fmaf(-0.5f, i3, 0.5f * i1);
      v[19] = fmaf(-0.25f, i2, 0.125f * i0);
      v[20] = fmaf(0.0625f, i8, fmaf(-0.25f, i6, 0.375f * i4));
      v[21] = fmaf(0.25f, i7, -0.75f * i5);
      v[22] = fmaf(0.125f, i8, fmaf(0.5f, i6, -1.25f * i4));
      v[23] = fmaf(0.75f, i7, 1.75f * i5);
      v[24] = fmaf(0.125f, i8, fmaf(3.5f, i6, 8.75f * i4));
    }
    {
      const float i0 = v[25]; const float i1 = v[26]; const float i2 = v[27]; const float i3 = v[28]; const float i4 = v[29]; const float i5 = v[30]; const float i6 = v[31]; const float i7 = v[32]; const float i8 = v[33]; const float i9 = v[34]; const float i10 = v[35];
      v[25] = fmaf(13.125f, i4, fmaf(2.8125f, i2, 0.0625f * i0));
      v[26] = fmaf(3.0f, i3, 0.5f * i1);
      v[27] = fmaf(-0.875f, i4, fmaf(0.8125f, i2, 0.0625f * i0));
      v[28] = fmaf(-0.5f, i3, 0.25f * i1);
      v[29] = fmaf(0.125f, i4, fmaf(-0.1875f, i2, 0.0625f * i0));
      v[30] = fmaf(0.03125f, i10, fmaf(-0.15625f, i8, 0.3125f * i6));
      v[31] = fmaf(0.125f, i9, fmaf(-0.5f, i7, 0.75f * i5));
      v[32] = fmaf(0.0625f, i10, fmaf(0.1875f, i8, -0.875f * i6));
      v[33] = fmaf(0.375f, i9, fmaf(0.5f, i7, -1.75f * i5));
      v[34] = fmaf(0.0625f, i10, fmaf(1.6875f, i8, 2.625f * i6));
      v[35] = fmaf(0.625f, i9, fmaf(7.5f, i7, 15.75f * i5));
    }
    {
      const float i0 = v[36]; const float i1 = v[37]; const float i2 = v[38]; const float i3 = v[39]; const float i4 = v[40]; const float i5 = v[41]; const float i6 = v[42]; const float i7 = v[43]; const float i8 = v[44]; const float i9 = v[45]; const float i10 = v[46]; const float i11 = v[47]; const float i12 = v[48];
      v[36] = fmaf(24.75f, i5, fmaf(6.875f, i3, 0.375f * i1));
      v[37] = fmaf(5.15625f, i4, fmaf(1.375f, i2, 0.03125f * i0));
      v[38] = fmaf(-1.5f, i5, fmaf(1.25f, i3, 0.25f * i1));
      v[39] = fmaf(-0.84375f, i4, fmaf(0.375f, i2, 0.03125f * i0));
      v[40] = fmaf(0.25f, i5, fmaf(-0.375f, i3, 0.125f * i1));
      v[41] = fmaf(0.15625f, i4, fmaf(-0.125f, i2, 0.03125f * i0));
      v[42] = fmaf(0.015625f, i12, fmaf(-0.09375f, i10, fmaf(0.234375f, i8, -0.3125f * i6)));
      v[43] = fmaf(0.0625f, i11, fmaf(-0.3125f, i9, 0.625f * i7));
      v[44] = fmaf(0.03125f, i12, fmaf(0.0625f, i10, fmaf(-0.53125f, i8, 0.875f * i6)));
      v[45] = fmaf(0.1875f, i11, fmaf(0.0625f, i9, -1.125f * i7));
      v[46] = fmaf(0.03125f, i12, fmaf(0.8125f, i10, fmaf(0.46875f, i8, -2.625f * i6)));
      v[47] = fmaf(0.3125f, i11, fmaf(3.4375f, i9, 4.125f * i7));
      v[48] = fmaf(0.03125f, i12, fmaf(2.0625f, i10, fmaf(15.46875f, i8, 28.875f * i6)));
    }
    {
      const float i0 = v[49]; const float i1 = v[50]; const float i2 = v[51]; const float i3 = v[52]; const float i4 = v[53]; const float i5 = v[54]; const float i6 = v[55]; const float i7 = v[56]; const float i8 = v[57]; const float i9 = v[58]; const float i10 = v[59]; const float i11 = v[60]; const float i12 = v[61]; const float i13 = v[62]; const float i14 = v[63];
      v[49] = fmaf(46.921875f, i6, fmaf(15.640625f, i4, fmaf(1.421875f, i2, 0.015625f * i0)));
      v[50] = fmaf(8.9375f, i5, fmaf(3.25f, i3, 0.1875f * i1));
      v[51] = fmaf(-2.578125f, i6, fmaf(1.890625f, i4, fmaf(0.671875f, i2, 0.015625f * i0)));
      v[52] = fmaf(-1.375f, i5, fmaf(0.5f, i3, 0.125f * i1));
      v[53] = fmaf(0.421875f, i6, fmaf(-0.609375f, i4, fmaf(0.171875f, i2, 0.015625f * i0)));
      v[54] = fmaf(0.3125f, i5, fmaf(-0.25f, i3, 0.0625f * i1));
      v[55] = fmaf(-0.078125f, i6, fmaf(0.140625f, i4, fmaf(-0.078125f, i2, 0.015625f * i0)));
      v[56] = fmaf(0.0078125f, i14, fmaf(-0.0546875f, i12, fmaf(0.1640625f, i10, -0.2734375f * i8)));
      v[57] = fmaf(0.03125f, i13, fmaf(-0.1875f, i11, fmaf(0.46875f, i9, -0.625f * i7)));
      v[58] = fmaf(0.015625f, i14, fmaf(0.015625f, i12, fmaf(-0.296875f, i10, 0.703125f * i8)));
      v[59] = fmaf(0.09375f, i13, fmaf(-0.0625f, i11, fmaf(-0.59375f, i9, 1.125f * i7)));
      v[60] = fmaf(0.015625f, i14, fmaf(0.390625f, i12, fmaf(-0.171875f, i10, -1.546875f * i8)));
      v[61] = fmaf(0.15625f, i13, fmaf(1.5625f, i11, fmaf(0.34375f, i9, -4.125f * i7)));
      v[62] = fmaf(0.015625f, i14, fmaf(1.015625f, i12, fmaf(6.703125f, i10, 6.703125f * i8)));
      v[63] = fmaf(0.21875f, i13, fmaf(5.6875f, i11, fmaf(31.28125f, i9, 53.625f * i7)));
    }
    {
      const float i0 = v[64]; const float i1 = v[65]; const float i2 = v[66]; const float i3 = v[67]; const float i4 = v[68]; const float i5 = v[69]; const float i6 = v[70]; const float i7 = v[71]; const float i8 = v[72]; const float i9 = v[73]; const float i10 = v[74]; const float i11 = v[75]; const float i12 = v[76]; const float i13 = v[77]; const float i14 = v[78]; const float i15 = v[79]; const float i16 = v[80];
      v[64] = fmaf(89.375f, i7, fmaf(34.125f, i5, fmaf(4.375f, i3, 0.125f * i1)));
      v[65] = fmaf(15.640625f, i6, fmaf(7.109375f, i4, fmaf(0.703125f, i2, 0.0078125f * i0)));
      v[66] = fmaf(-4.46875f, i7, fmaf(2.84375f, i5, fmaf(1.53125f, i3, 0.09375f * i1)));
      v[67] = fmaf(-2.234375f, i6, fmaf(0.609375f, i4, fmaf(0.328125f, i2, 0.0078125f * i0)));
      v[68] = fmaf(0.6875f, i7, fmaf(-0.9375f, i5, fmaf(0.1875f, i3, 0.0625f * i1)));
      v[69] = fmaf(0.515625f, i6, fmaf(-0.390625f, i4, fmaf(0.078125f, i2, 0.0078125f * i0)));
      v[70] = fmaf(-0.15625f, i7, fmaf(0.28125f, i5, fmaf(-0.15625f, i3, 0.03125f * i1)));
      v[71] = fmaf(-0.109375f, i6, fmaf(0.109375f, i4, fmaf(-0.046875f, i2, 0.0078125f * i0)));
      v[72] = fmaf(0.00390625f, i16, fmaf(-0.03125f, i14, fmaf(0.109375f, i12, fmaf(-0.21875f, i10, 0.2734375f * i8))));
      v[73] = fmaf(0.015625f, i15, fmaf(-0.109375f, i13, fmaf(0.328125f, i11, -0.546875f * i9)));
      v[74] = fmaf(0.0078125f, i16, fmaf(-0.15625f, i12, fmaf(0.5f, i10, -0.703125f * i8)));
      v[75] = fmaf(0.046875f, i15, fmaf(-0.078125f, i13, fmaf(-0.265625f, i11, 0.859375f * i9)));
      v[76] = fmaf(0.0078125f, i16, fmaf(0.1875f, i14, fmaf(-0.28125f, i12, fmaf(-0.6875f, i10, 1.546875f * i8))));
      v[77] = fmaf(0.078125f, i15, fmaf(0.703125f, i13, fmaf(-0.609375f, i11, -2.234375f * i9)));
      v[78] = fmaf(0.0078125f, i16, fmaf(0.5f, i14, fmaf(2.84375f, i12, -6.703125f * i8)));
      v[79] = fmaf(0.109375f, i15, fmaf(2.734375f, i13, fmaf(12.796875f, i11, 11.171875f * i9)));
      v[80] = fmaf(0.0078125f, i16, fmaf(0.9375f, i14, fmaf(14.21875f, i12, fmaf(62.5625f, i10, 100.546875f * i8))));
    }
    {
      const float i0 = v[81]; const float i1 = v[82]; const float i2 = v[83]; const float i3 = v[84]; const float i4 = v[85]; const float i5 = v[86]; const float i6 = v[87]; const float i7 = v[88]; const float i8 = v[89]; const float i9 = v[90]; const float i10 = v[91]; const float i11 = v[92]; const float i12 = v[93]; const float i13 = v[94]; const float i14 = v[95]; const float i15 = v[96]; const float i16 = v[97]; const float i17 = v[98]; const float i18 = v[99];
      v[81] = fmaf(170.9296875f, i8, fmaf(72.515625f, i6, fmaf(11.953125f, i4, fmaf(0.59765625f, i2, 0.00390625f * i0))));
      v[82] = fmaf(27.625f, i7, fmaf(14.875f, i5, fmaf(2.125f, i3, 0.0625f * i1)));
      v[83] = fmaf(-7.8203125f, i8, fmaf(4.265625f, i6, fmaf(3.203125f, i4, fmaf(0.34765625f, i2, 0.00390625f * i0))));
      v[84] = fmaf(-3.65625f, i7, fmaf(0.65625f, i5, fmaf(0.71875f, i3, 0.046875f * i1)));
      v[85] = fmaf(1.1171875f, i8, fmaf(-1.421875f, i6, fmaf(0.140625f, i4, fmaf(0.16015625f, i2, 0.00390625f * i0))));
      v[86] = fmaf(0.8125f, i7, fmaf(-0.5625f, i5, fmaf(0.0625f, i3, 0.03125f * i1)));
      v[87] = fmaf(-0.2578125f, i8, fmaf(0.453125f, i6, fmaf(-0.234375f, i4, fmaf(0.03515625f, i2, 0.00390625f * i0))));
      v[88] = fmaf(-0.21875f, i7, fmaf(0.21875f, i5, fmaf(-0.09375f, i3, 0.015625f * i1)));
      v[89] = fmaf(0.0546875f, i8, fmaf(-0.109375f, i6, fmaf(0.078125f, i4, fmaf(-0.02734375f, i2, 0.00390625f * i0))));
      v[90] = fmaf(0.001953125f, i18, fmaf(-0.017578125f, i16, fmaf(0.0703125f, i14, fmaf(-0.1640625f, i12, 0.24609375f * i10))));
      v[91] = fmaf(0.0078125f, i17, fmaf(-0.0625f, i15, fmaf(0.21875f, i13, fmaf(-0.4375f, i11, 0.546875f * i9))));
      v[92] = fmaf(0.00390625f, i18, fmaf(-0.00390625f, i16, fmaf(-0.078125f, i14, fmaf(0.328125f, i12, -0.6015625f * i10))));
      v[93] = fmaf(0.0234375f, i17, fmaf(-0.0625f, i15, fmaf(-0.09375f, i13, fmaf(0.5625f, i11, -0.859375f * i9))));
      v[94] = fmaf(0.00390625f, i18, fmaf(0.08984375f, i16, fmaf(-0.234375f, i14, fmaf(-0.203125f, i12, 1.1171875f * i10))));
      v[95] = fmaf(0.0390625f, i17, fmaf(0.3125f, i15, fmaf(-0.65625f, i13, fmaf(-0.8125f, i11, 2.234375f * i9))));
      v[96] = fmaf(0.00390625f, i18, fmaf(0.24609375f, i16, fmaf(1.171875f, i14, fmaf(-1.421875f, i12, -3.3515625f * i10))));
      v[97] = fmaf(0.0546875f, i17, fmaf(1.3125f, i15, fmaf(5.03125f, i13, fmaf(-0.8125f, i11, -11.171875f * i9))));
      v[98] = fmaf(0.00390625f, i18, fmaf(0.46484375f, i16, fmaf(6.640625f, i14, fmaf(24.171875f, i12, 18.9921875f * i10))));
      v[99] = fmaf(0.0703125f, i17, fmaf(3.1875f, i15, fmaf(33.46875f, i13, fmaf(124.3125f, i11, 189.921875f * i9))));
    }
  }
};
template <> struct BApply<10, false> {
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[1]; const float i1 = v[2]; const float i2 = v[3];
      v[1] = 1.0f * i0;
      v[2] = 2.0f * i2;
      v[3] = 0.5f * i1;
    }
    {
      const float i0 = v[4]; const float i1 = v[5]; const float i2 = v[6]; const float i3 = v[7]; const float i4 = v[8];
      v[4] = 0.5f * i1;
      v[5] = 2.0f * i0;
      v[6] = fmaf(3.0f, i4, -0.5f * i2);
      v[7] = 1.0f * i3;
      v[8] = fmaf(0.5f, i4, 0.25f * i2);
    }
    {
      const float i0 = v[9]; const float i1 = v[10]; const float i2 = v[11]; const float i3 = v[12]; const float i4 = v[13]; const float i5 = v[14]; const float i6 = v[15];
      v[9] = fmaf(0.25f, i2, 0.25f * i0);
      v[10] = 1.0f * i1;
      v[11] = fmaf(-0.25f, i2, 3.75f * i0);
      v[12] = fmaf(5.0f, i6, -1.0f * i4);
      v[13] = fmaf(1.25f, i5, -0.375f * i3);
      v[14] = fmaf(1.5f, i6, 0.5f * i4);
      v[15] = fmaf(0.25f, i5, 0.125f * i3);
    }
    {
      const float i0 = v[16]; const float i1 = v[17]; const float i2 = v[18]; const float i3 = v[19]; const float i4 = v[20]; const float i5 = v[21]; const float i6 = v[22]; const float i7 = v[23]; const float i8 = v[24];
      v[16] = fmaf(0.125f, i3, 0.125f * i1);
      v[17] = fmaf(0.5f, i2, 1.0f * i0);
      v[18] = fmaf(-0.25f, i3, 1.75f * i1);
      v[19] = fmaf(-0.5f, i2, 7.0f * i0);
      v[20] = fmaf(8.75f, i8, fmaf(-1.25f, i6, 0.375f * i4));
      v[21] = fmaf(1.75f, i7, -0.75f * i5);
      v[22] = fmaf(3.5f, i8, fmaf(0.5f, i6, -0.25f * i4));
      v[23] = fmaf(0.75f, i7, 0.25f * i5);
      v[24] = fmaf(0.125f, i8, fmaf(0.125f, i6, 0.0625f * i4));
    }
    {
      const float i0 = v[25]; const float i1 = v[26]; const float i2 = v[27]; const float i3 = v[28]; const float i4 = v[29]; const float i5 = v[30]; const float i6 = v[31]; const float i7 = v[32]; const float i8 = v[33]; const float i9 = v[34]; const float i10 = v[35];
      v[25] = fmaf(0.0625f, i4, fmaf(0.0625f, i2, 0.0625f * i0));
      v[26] = fmaf(0.25f, i3, 0.5f * i1);
      v[27] = fmaf(-0.1875f, i4, fmaf(0.8125f, i2, 2.8125f * i0));
      v[28] = fmaf(-0.5f, i3, 3.0f * i1);
      v[29] = fmaf(0.125f, i4, fmaf(-0.875f, i2, 13.125f * i0));
      v[30] = fmaf(15.75f, i10, fmaf(-1.75f, i8, 0.75f * i6));
      v[31] = fmaf(2.625f, i9, fmaf(-0.875f, i7, 0.3125f * i5));
      v[32] = fmaf(7.5f, i10, fmaf(0.5f, i8, -0.5f * i6));
      v[33] = fmaf(1.6875f, i9, fmaf(0.1875f, i7, -0.15625f * i5));
      v[34] = fmaf(0.625f, i10, fmaf(0.375f, i8, 0.125f * i6));
      v[35] = fmaf(0.0625f, i9, fmaf(0.0625f, i7, 0.03125f * i5));
    }
    {
      const float i0 = v[36]; const float i1 = v[37]; const float i2 = v[38]; const float i3 = v[39]; const float i4 = v[40]; const float i5 = v[41]; const float i6 = v[42]; const float i7 = v[43]; const float i8 = v[44]; const float i9 = v[45]; const float i10 = v[46]; const float i11 = v[47]; const float i12 = v[48];
      v[36] = fmaf(0.03125f, i5, fmaf(0.03125f, i3, 0.03125f * i1));
      v[37] = fmaf(0.125f, i4, fmaf(0.25f, i2, 0.375f * i0));
      v[38] = fmaf(-0.125f, i5, fmaf(0.375f, i3, 1.375f * i1));
      v[39] = fmaf(-0.375f, i4, fmaf(1.25f, i2, 6.875f * i0));
      v[40] = fmaf(0.15625f, i5, fmaf(-0.84375f, i3, 5.15625f * i1));
      v[41] = fmaf(0.25f, i4, fmaf(-1.5f, i2, 24.75f * i0));
      v[42] = fmaf(28.875f, i12, fmaf(-2.625f, i10, fmaf(0.875f, i8, -0.3125f * i6)));
      v[43] = fmaf(4.125f, i11, fmaf(-1.125f, i9, 0.625f * i7));
      v[44] = fmaf(15.46875f, i12, fmaf(0.46875f, i10, fmaf(-0.53125f, i8, 0.234375f * i6)));
      v[45] = fmaf(3.4375f, i11, fmaf(0.0625f, i9, -0.3125f * i7));
      v[46] = fmaf(2.0625f, i12, fmaf(0.8125f, i10, fmaf(0.0625f, i8, -0.09375f * i6)));
      v[47] = fmaf(0.3125f, i11, fmaf(0.1875f, i9, 0.0625f * i7));
      v[48] = fmaf(0.03125f, i12, fmaf(0.03125f, i10, fmaf(0.03125f, i8, 0.015625f * i6)));
    }
    {
      const float i0 = v[49]; const float i1 = v[50]; const float i2 = v[51]; const float i3 = v[52]; const float i4 = v[53]; const float i5 = v[54]; const float i6 = v[55]; const float i7 = v[56]; const float i8 = v[57]; const float i9 = v[58]; const float i10 = v[59]; const float i11 = v[60]; const float i12 = v[61]; const float i13 = v[62]; const float i14 = v[63];
      v[49] = fmaf(0.015625f, i6, fmaf(0.015625f, i4, fmaf(0.015625f, i2, 0.015625f * i0)));
      v[50] = fmaf(0.0625f, i5, fmaf(0.125f, i3, 0.1875f * i1));
      v[51] = fmaf(-0.078125f, i6, fmaf(0.171875f, i4, fmaf(0.671875f, i2, 1.421875f * i0)));
      v[52] = fmaf(-0.25f, i5, fmaf(0.5f, i3, 3.25f * i1));
      v[53] = fmaf(0.140625f, i6, fmaf(-0.609375f, i4, fmaf(1.890625f, i2, 15.640625f * i0)));
      v[54] = fmaf(0.3125f, i5, fmaf(-1.375f, i3, 8.9375f * i1));
      v[55] = fmaf(-0.078125f, i6, fmaf(0.421875f, i4, fmaf(-2.578125f, i2, 46.921875f * i0)));
      v[56] = fmaf(53.625f, i14, fmaf(-4.125f, i12, fmaf(1.125f, i10, -0.625f * i8)));
      v[57] = fmaf(6.703125f, i13, fmaf(-1.546875f, i11, fmaf(0.703125f, i9, -0.2734375f * i7)));
      v[58] = fmaf(31.28125f, i14, fmaf(0.34375f, i12, fmaf(-0.59375f, i10, 0.46875f * i8)));
      v[59] = fmaf(6.703125f, i13, fmaf(-0.171875f, i11, fmaf(-0.296875f, i9, 0.1640625f * i7)));
      v[60] = fmaf(5.6875f, i14, fmaf(1.5625f, i12, fmaf(-0.0625f, i10, -0.1875f * i8)));
      v[61] = fmaf(1.015625f, i13, fmaf(0.390625f, i11, fmaf(0.015625f, i9, -0.0546875f * i7)));
      v[62] = fmaf(0.21875f, i14, fmaf(0.15625f, i12, fmaf(0.09375f, i10, 0.03125f * i8)));
      v[63] = fmaf(0.015625f, i13, fmaf(0.015625f, i11, fmaf(0.015625f, i9, 0.0078125f * i7)));
    }
    {
      const float i0 = v[64]; const float i1 = v[65]; const float i2 = v[66]; const float i3 = v[67]; const float i4 = v[68]; const float i5 = v[69]; const float i6 = v[70]; const float i7 = v[71]; const float i8 = v[72]; const float i9 = v[73]; const float i10 = v[74]; const float i11 = v[75]; const float i12 = v[76]; const float i13 = v[77]; const float i14 = v[78]; const float i15 = v[79]; const float i16 = v[80];
      v[64] = fmaf(0.0078125f, i7, fmaf(0.0078125f, i5, fmaf(0.0078125f, i3, 0.0078125f * i1)));
      v[65] = fmaf(0.03125f, i6, fmaf(0.0625f, i4, fmaf(0.09375f, i2, 0.125f * i0)));
      v[66] = fmaf(-0.046875f, i7, fmaf(0.078125f, i5, fmaf(0.328125f, i3, 0.703125f * i1)));
      v[67] = fmaf(-0.15625f, i6, fmaf(0.1875f, i4, fmaf(1.53125f, i2, 4.375f * i0)));
      v[68] = fmaf(0.109375f, i7, fmaf(-0.390625f, i5, fmaf(0.609375f, i3, 7.109375f * i1)));
      v[69] = fmaf(0.28125f, i6, fmaf(-0.9375f, i4, fmaf(2.84375f, i2, 34.125f * i0)));
      v[70] = fmaf(-0.109375f, i7, fmaf(0.515625f, i5, fmaf(-2.234375f, i3, 15.640625f * i1)));
      v[71] = fmaf(-0.15625f, i6, fmaf(0.6875f, i4, fmaf(-4.46875f, i2, 89.375f * i0)));
      v[72] = fmaf(100.546875f, i16, fmaf(-6.703125f, i14, fmaf(1.546875f, i12, fmaf(-0.703125f, i10, 0.2734375f * i8))));
      v[73] = fmaf(11.171875f, i15, fmaf(-2.234375f, i13, fmaf(0.859375f, i11, -0.546875f * i9)));
      v[74] = fmaf(62.5625f, i16, fmaf(-0.6875f, i12, fmaf(0.5f, i10, -0.21875f * i8)));
      v[75] = fmaf(12.796875f, i15, fmaf(-0.609375f, i13, fmaf(-0.265625f, i11, 0.328125f * i9)));
      v[76] = fmaf(14.21875f, i16, fmaf(2.84375f, i14, fmaf(-0.28125f, i12, fmaf(-0.15625f, i10, 0.109375f * i8))));
      v[77] = fmaf(2.734375f, i15, fmaf(0.703125f, i13, fmaf(-0.078125f, i11, -0.109375f * i9)));
      v[78] = fmaf(0.9375f, i16, fmaf(0.5f, i14, fmaf(0.1875f, i12, -0.03125f * i8)));
      v[79] = fmaf(0.109375f, i15, fmaf(0.078125f, i13, fmaf(0.046875f, i11, 0.015625f * i9)));
      v[80] = fmaf(0.0078125f, i16, fmaf(0.0078125f, i14, fmaf(0.0078125f, i12, fmaf(0.0078125f, i10, 0.00390625f * i8))));
    }
    {
      const float i0 = v[81]; const float i1 = v[82]; const float i2 = v[83]; const float i3 = v[84]; const float i4 = v[85]; const float i5 = v[86]; const float i6 = v[87]; const float i7 = v[88]; const float i8 = v[89]; const float i9 = v[90]; const float i10 = v[91]; const float i11 = v[92]; const float i12 = v[93]; const float i13 = v[94]; const float i14 = v[95]; const float i15 = v[96]; const float i16 = v[97]; const float i17 = v[98]; const float i18 = v[99];
      v[81] = fmaf(0.00390625f, i8, fmaf(0.00390625f, i6, fmaf(0.00390625f, i4, fmaf(0.00390625f, i2, 0.00390625f * i0))));
      v[82] = fmaf(0.015625f, i7, fmaf(0.03125f, i5, fmaf(0.046875f, i3, 0.0625f * i1)));
      v[83] = fmaf(-0.02734375f, i8, fmaf(0.03515625f, i6, fmaf(0.16015625f, i4, fmaf(0.34765625f, i2, 0.59765625f * i0))));
      v[84] = fmaf(-0.09375f, i7, fmaf(0.0625f, i5, fmaf(0.71875f, i3, 2.125f * i1)));
      v[85] = fmaf(0.078125f, i8, fmaf(-0.234375f, i6, fmaf(0.140625f, i4, fmaf(3.203125f, i2, 11.953125f * i0))));
      v[86] = fmaf(0.21875f, i7, fmaf(-0.5625f, i5, fmaf(0.65625f, i3, 14.875f * i1)));
      v[87] = fmaf(-0.109375f, i8, fmaf(0.453125f, i6, fmaf(-1.421875f, i4, fmaf(4.265625f, i2, 72.515625f * i0))));
      v[88] = fmaf(-0.21875f, i7, fmaf(0.8125f, i5, fmaf(-3.65625f, i3, 27.625f * i1)));
      v[89] = fmaf(0.0546875f, i8, fmaf(-0.2578125f, i6, fmaf(1.1171875f, i4, fmaf(-7.8203125f, i2, 170.9296875f * i0))));
      v[90] = fmaf(189.921875f, i18, fmaf(-11.171875f, i16, fmaf(2.234375f, i14, fmaf(-0.859375f, i12, 0.546875f * i10))));
      v[91] = fmaf(18.9921875f, i17, fmaf(-3.3515625f, i15, fmaf(1.1171875f, i13, fmaf(-0.6015625f, i11, 0.24609375f * i9))));
      v[92] = fmaf(124.3125f, i18, fmaf(-0.8125f, i16, fmaf(-0.8125f, i14, fmaf(0.5625f, i12, -0.4375f * i10))));
      v[93] = fmaf(24.171875f, i17, fmaf(-1.421875f, i15, fmaf(-0.203125f, i13, fmaf(0.328125f, i11, -0.1640625f * i9))));
      v[94] = fmaf(33.46875f, i18, fmaf(5.03125f, i16, fmaf(-0.65625f, i14, fmaf(-0.09375f, i12, 0.21875f * i10))));
      v[95] = fmaf(6.640625f, i17, fmaf(1.171875f, i15, fmaf(-0.234375f, i13, fmaf(-0.078125f, i11, 0.0703125f * i9))));
      v[96] = fmaf(3.1875f, i18, fmaf(1.3125f, i16, fmaf(0.3125f, i14, fmaf(-0.0625f, i12, -0.0625f * i10))));
      v[97] = fmaf(0.46484375f, i17, fmaf(0.24609375f, i15, fmaf(0.08984375f, i13, fmaf(-0.00390625f, i11, -0.017578125f * i9))));
      v[98] = fmaf(0.0703125f, i18, fmaf(0.0546875f, i16, fmaf(0.0390625f, i14, fmaf(0.0234375f, i12, 0.0078125f * i10))));
      v[99] = fmaf(0.00390625f, i17, fmaf(0.00390625f, i15, fmaf(0.00390625f, i13, fmaf(0.00390625f, i11, 0.001953125f * i9))));
    }
    {
      const float i0 = v[100]; const float i1 = v[101]; const float i2 = v[102]; const float i3 = v[103]; const float i4 = v[104]; const float i5 = v[105]; const float i6 = v[106]; const float i7 = v[107]; const float i8 = v[108]; const float i9 = v[109]; const float i10 = v[110]; const float i11 = v[111]; const float i12 = v[112]; const float i13 = v[113]; const float i14 = v[114]; const float i15 = v[115]; const float i16 = v[116]; const float i17 = v[117]; const float i18 = v[118]; const float i19 = v[119]; const float i20 = v[120];
      v[100] = fmaf(0.001953125f, i9, fmaf(0.001953125f, i7, fmaf(0.001953125f, i5, fmaf(0.001953125f, i3, 0.001953125f * i1))));
      v[101] = fmaf(0.0078125f, i8, fmaf(0.015625f, i6, fmaf(0.0234375f, i4, fmaf(0.03125f, i2, 0.0390625f * i0))));
      v[102] = fmaf(-0.015625f, i9, fmaf(0.015625f, i7, fmaf(0.078125f, i5, fmaf(0.171875f, i3, 0.296875f * i1))));
      v[103] = fmaf(-0.0546875f, i8, fmaf(0.015625f, i6, fmaf(0.3359375f, i4, fmaf(1.03125f, i2, 2.2265625f * i0))));
      v[104] = fmaf(0.052734375f, i9, fmaf(-0.134765625f, i7, fmaf(-0.009765625f, i5, fmaf(1.427734375f, i3, 5.677734375f * i1))));
      v[105] = fmaf(0.15625f, i8, fmaf(-0.3125f, i6, fmaf(-0.03125f, i4, fmaf(6.375f, i2, 30.28125f * i0))));
      v[106] = fmaf(-0.09375f, i9, fmaf(0.34375f, i7, fmaf(-0.78125f, i5, fmaf(0.53125f, i3, 30.28125f * i1))));
      v[107] = fmaf(-0.21875f, i8, fmaf(0.6875f, i6, fmaf(-2.15625f, i4, fmaf(6.375f, i2, 151.40625f * i0))));
      v[108] = fmaf(0.08203125f, i9, fmaf(-0.35546875f, i7, fmaf(1.26953125f, i5, fmaf(-6.04296875f, i3, 49.20703125f * i1))));
      v[109] = fmaf(0.109375f, i8, fmaf(-0.40625f, i6, fmaf(1.828125f, i4, fmaf(-13.8125f, i2, 328.046875f * i0))));
      v[110] = fmaf(360.8515625f, i20, fmaf(-18.9921875f, i18, fmaf(3.3515625f, i16, fmaf(-1.1171875f, i14, fmaf(0.6015625f, i12, -0.24609375f * i10)))));
      v[111] = fmaf(32.8046875f, i19, fmaf(-5.1796875f, i17, fmaf(1.5234375f, i15, fmaf(-0.7109375f, i13, 0.4921875f * i11))));
      v[112] = fmaf(246.03515625f, i20, fmaf(-2.58984375f, i18, fmaf(-0.96484375f, i16, fmaf(0.66015625f, i14, fmaf(-0.46484375f, i12, 0.205078125f * i10)))));
      v[113] = fmaf(45.421875f, i19, fmaf(-2.921875f, i17, fmaf(-0.078125f, i15, fmaf(0.328125f, i13, -0.328125f * i11))));
      v[114] = fmaf(75.703125f, i20, fmaf(8.765625f, i18, fmaf(-1.296875f, i16, fmaf(0.015625f, i14, fmaf(0.203125f, i12, -0.1171875f * i10)))));
      v[115] = fmaf(15.140625f, i19, fmaf(1.859375f, i17, fmaf(-0.484375f, i15, fmaf(-0.015625f, i13, 0.140625f * i11))));
      v[116] = fmaf(9.462890625f, i20, fmaf(3.087890625f, i18, fmaf(0.462890625f, i16, fmaf(-0.162109375f, i14, fmaf(-0.037109375f, i12, 0.0439453125f * i10)))));
      v[117] = fmaf(1.55859375f, i19, fmaf(0.62890625f, i17, fmaf(0.13671875f, i15, fmaf(-0.04296875f, i13, -0.03515625f * i11))));
      v[118] = fmaf(0.37109375f, i20, fmaf(0.23046875f, i18, fmaf(0.12109375f, i16, fmaf(0.04296875f, i14, fmaf(-0.00390625f, i12, -0.009765625f * i10)))));
      v[119] = fmaf(0.03515625f, i19, fmaf(0.02734375f, i17, fmaf(0.01953125f, i15, fmaf(0.01171875f, i13, 0.00390625f * i11))));
      v[120] = fmaf(0.001953125f, i20, fmaf(0.001953125f, i18, fmaf(0.001953125f, i16, fmaf(0.001953125f, i14, fmaf(0.001953125f, i12, 0.0009765625f * i10)))));
    }
  }
};
template <> struct BApply<10, true> {
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[1]; const float i1 = v[2]; const float i2 = v[3];
      v[1] = 1.0f * i0;
      v[2] = 0.5f * i2;
      v[3] = 2.0f * i1;
    }
    {
      const float i0 = v[4]; const float i1 = v[5]; const float i2 = v[6]; const float i3 = v[7]; const float i4 = v[8];
      v[4] = 2.0f * i1;
      v[5] = 0.5f * i0;
      v[6] = fmaf(0.25f, i4, -0.5f * i2);
      v[7] = 1.0f * i3;
      v[8] = fmaf(0.5f, i4, 3.0f * i2);
    }
    {
      const float i0 = v[9]; const float i1 = v[10]; const float i2 = v[11]; const float i3 = v[12]; const float i4 = v[13]; const float i5 = v[14]; const float i6 = v[15];
      v[9] = fmaf(3.75f, i2, 0.25f * i0);
      v[10] = 1.0f * i1;
      v[11] = fmaf(-0.25f, i2, 0.25f * i0);
      v[12] = fmaf(0.125f, i6, -0.375f * i4);
      v[13] = fmaf(0.5f, i5, -1.0f * i3);
      v[14] = fmaf(0.25f, i6, 1.25f * i4);
      v[15] = fmaf(1.5f, i5, 5.0f * i3);
    }
    {
      const float i0 = v[16]; const float i1 = v[17]; const float i2 = v[18]; const float i3 = v[19]; const float i4 = v[20]; const float i5 = v[21]; const float i6 = v[22]; const float i7 = v[23]; const float i8 = v[24];
      v[16] = fmaf(7.0f, i3, 1.0f * i1);
      v[17] = fmaf(1.75f, i2, 0.125f * i0);
      v[18] = fmaf(-0.5f, i3, 0.5f * i1);
      v[19] = fmaf(-0.25f, i2, 0.125f * i0);
      v[20] = fmaf(0.0625f, i8, fmaf(-0.25f, i6, 0.375f * i4));
      v[21] = fmaf(0.25f, i7, -0.75f * i5);
      v[22] = fmaf(0.125f, i8, fmaf(0.5f, i6, -1.25f * i4));
      v[23] = fmaf(0.75f, i7, 1.75f * i5);
      v[24] = fmaf(0.125f, i8, fmaf(3.5f, i6, 8.75f * i4));
    }
    {
      const float i0 = v[25]; const float i1 = v[26]; const float i2 = v[27]; const float i3 = v[28]; const float i4 = v[29]; const float i5 = v[30]; const float i6 = v[31]; const float i7 = v[32]; const float i8 = v[33]; const float i9 = v[34]; const float i10 = v[35];
      v[25] = fmaf(13.125f, i4, fmaf(2.8125f, i2, 0.0625f * i0));
      v[26] = fmaf(3.0f, i3, 0.5f * i1);
      v[27] = fmaf(-0.875f, i4, fmaf(0.8125f, i2, 0.0625f * i0));
      v[28] = fmaf(-0.5f, i3, 0.25f * i1);
      v[29] = fmaf(0.125f, i4, fmaf(-0.1875f, i2, 0.0625f * i0));
      v[30] = fmaf(0.03125f, i10, fmaf(-0.15625f, i8, 0.3125f * i6));
      v[31] = fmaf(0.125f, i9, fmaf(-0.5f, i7, 0.75f * i5));
      v[32] = fmaf(0.0625f, i10, fmaf(0.1875f, i8, -0.875f * i6));
      v[33] = fmaf(0.375f, i9, fmaf(0.5f, i7, -1.75f * i5));
      v[34] = fmaf(0.0625f, i10, fmaf(1.6875f, i8, 2.625f * i6));
      v[35] = fmaf(0.625f, i9, fmaf(7.5f, i7, 15.75f * i5));
    }
    {
      const float i0 = v[36]; const float i1 = v[37]; const float i2 = v[38]; const float i3 = v[39]; const float i4 = v[40]; const float i5 = v[41]; const float i6 = v[42]; const float i7 = v[43]; const float i8 = v[44]; const float i9 = v[45]; const float i10 = v[46]; const float i11 = v[47]; const float i12 = v[48];
      v[36] = fmaf(24.75f, i5, fmaf(6.875f, i3, 0.375f * i1));
      v[37] = fmaf(5.15625f, i4, fmaf(1.375f, i2, 0.03125f * i0));
      v[38] = fmaf(-1.5f, i5, fmaf(1.25f, i3, 0.25f * i1));
      v[39] = fmaf(-0.84375f, i4, fmaf(0.375f, i2, 0.03125f * i0));
      v[40] = fmaf(0.25f, i5, fmaf(-0.375f, i3, 0.125f * i1));
      v[41] = fmaf(0.15625f, i4, fmaf(-0.125f, i2, 0.03125f * i0));
      v[42] = fmaf(0.015625f, i12, fmaf(-0.09375f, i10, fmaf(0.234375f, i8, -0.3125f * i6)));
      v[43] = fmaf(0.0625f, i11, fmaf(-0.3125f, i9, 0.625f * i7));
      v[44] = fmaf(0.03125f, i12, fmaf(0.0625f, i10, fmaf(-0.53125f, i8, 0.875f * i6)));
      v[45] = fmaf(0.1875f, i11, fmaf(0.0625f, i9, -1.125f * i7));
      v[46] = fmaf(0.03125f, i12, fmaf(0.8125f, i10, fmaf(0.46875f, i8, -2.625f * i6)));
      v[47] = fmaf(0.3125f, i11, fmaf(3.4375f, i9, 4.125f * i7));
      v[48] = fmaf(0.03125f, i12, fmaf(2.0625f, i10, fmaf(15.46875f, i8, 28.875f * i6)));
    }
    {
      const float i0 = v[49]; const float i1 = v[50]; const float i2 = v[51]; const float i3 = v[52]; const float i4 = v[53]; const float i5 = v[54]; const float i6 = v[55]; const float i7 = v[56]; const float i8 = v[57]; const float i9 = v[58]; const float i10 = v[59]; const float i11 = v[60]; const float i12 = v[61]; const float i13 = v[62]; const float i14 = v[63];
      v[49] = fmaf(46.921875f, i6, fmaf(15.640625f, i4, fmaf(1.421875f, i2, 0.015625f * i0)));
      v[50] = fmaf(8.9375f, i5, fmaf(3.25f, i3, 0.1875f * i1));
      v[51] = fmaf(-2.578125f, i6, fmaf(1.890625f, i4, fmaf(0.671875f, i2, 0.015625f * i0)));
      v[52] = fmaf(-1.375f, i5, fmaf(0.5f, i3, 0.125f * i1));
      v[53] = fmaf(0.421875f, i6, fmaf(-0.609375f, i4, fmaf(0.171875f, i2, 0.015625f * i0)));
      v[54] = fmaf(0.3125f, i5, fmaf(-0.25f, i3, 0.0625f * i1));
      v[55] = fmaf(-0.078125f, i6, fmaf(0.140625f, i4, fmaf(-0.078125f, i2, 0.015625f * i0)));
      v[56] = fmaf(0.0078125f, i14, fmaf(-0.0546875f, i12, fmaf(0.1640625f, i10, -0.2734375f * i8)));
      v[57] = fmaf(0.03125f, i13, fmaf(-0.1875f, i11, fmaf(0.46875f, i9, -0.625f * i7)));
      v[58] = fmaf(0.015625f, i14, fmaf(0.015625f, i12, fmaf(-0.296875f, i10, 0.703125f * i8)));
      v[59] = fmaf(0.09375f, i13, fmaf(-0.0625f, i11, fmaf(-0.59375f, i9, 1.125f * i7)));
      v[60] = fmaf(0.015625f, i14, fmaf(0.390625f, i12, fmaf(-0.171875f, i10, -1.546875f * i8)));
      v[61] = fmaf(0.15625f, i13, fmaf(1.5625f, i11, fmaf(0.34375f, i9, -4.125f * i7)));
      v[62] = fmaf(0.015625f, i14, fmaf(1.015625f, i12, fmaf(6.703125f, i10, 6.703125f * i8)));
      v[63] = fmaf(0.21875f, i13, fmaf(5.6875f, i11, fmaf(31.28125f, i9, 53.625f * i7)));
    }
    {
      const float i0 = v[64]; const float i1 = v[65]; const float i2 = v[66]; const float i3 = v[67]; const float i4 = v[68]; const float i5 = v[69]; const float i6 = v[70]; const float i7 = v[71]; const float i8 = v[72]; const float i9 = v[73]; const float i10 = v[74]; const float i11 = v[75]; const float i12 = v[76]; const float i13 = v[77]; const float i14 = v[78]; const float i15 = v[79]; const float i16 = v[80];
      v[64] = fmaf(89.375f, i7, fmaf(34.125f, i5, fmaf(4.375f, i3, 0.125f * i1)));
      v[65] = fmaf(15.640625f, i6, fmaf(7.109375f, i4, fmaf(0.703125f, i2, 0.0078125f * i0)));
      v[66] = fmaf(-4.46875f, i7, fmaf(2.84375f, i5, fmaf(1.53125f, i3, 0.09375f * i1)));
      v[67] = fmaf(-2.234375f, i6, fmaf(0.609375f, i4, fmaf(0.328125f, i2, 0.0078125f * i0)));
      v[68] = fmaf(0.6875f, i7, fmaf(-0.9375f, i5, fmaf(0.1875f, i3, 0.0625f * i1)));
      v[69] = fmaf(0.515625f, i6, fmaf(-0.390625f, i4, fmaf(0.078125f, i2, 0.0078125f * i0)));
      v[70] = fmaf(-0.15625f, i7, fmaf(0.28125f, i5, fmaf(-0.15625f, i3, 0.03125f * i1)));
      v[71] = fmaf(-0.109375f, i6, fmaf(0.109375f, i4, fmaf(-0.046875f, i2, 0.0078125f * i0)));
      v[72] = fmaf(0.00390625f, i16, fmaf(-0.03125f, i14, fmaf(0.109375f, i12, fmaf(-0.21875f, i10, 0.2734375f * i8))));
      v[73] = fmaf(0.015625f, i15, fmaf(-0.109375f, i13, fmaf(0.328125f, i11, -0.546875f * i9)));
      v[74] = fmaf(0.0078125f, i16, fmaf(-0.15625f, i12, fmaf(0.5f, i10, -0.703125f * i8)));
      v[75] = fmaf(0.046875f, i15, fmaf(-0.078125f, i13, fmaf(-0.265625f, i11, 0.859375f * i9)));
      v[76] = fmaf(0.0078125f, i16, fmaf(0.1875f, i14, fmaf(-0.28125f, i12, fmaf(-0.6875f, i10, 1.546875f * i8))));
      v[77] = fmaf(0.078125f, i15, fmaf(0.703125f, i13, fmaf(-0.609375f, i11, -2.234375f * i9)));
      v[78] = fmaf(0.0078125f, i16, fmaf(0.5f, i14, fmaf(2.84375f, i12, -6.703125f * i8)));
      v[79] = fmaf(0.109375f, i15, fmaf(2.734375f, i13, fmaf(12.796875f, i11, 11.171875f * i9)));
      v[80] = fmaf(0.0078125f, i16, fmaf(0.9375f, i14, fmaf(14.21875f, i12, fmaf(62.5625f, i10, 100.546875f * i8))));
    }
    {
      const float i0 = v[81]; const float i1 = v[82]; const float i2 = v[83]; const float i3 = v[84]; const float i4 = v[85]; const float i5 = v[86]; const float i6 = v[87]; const float i7 = v[88]; const float i8 = v[89]; const float i9 = v[90]; const float i10 = v[91]; const float i11 = v[92]; const float i12 = v[93]; const float i13 = v[94]; const float i14 = v[95]; const float i15 = v[96]; const float i16 = v[97]; const float i17 = v[98]; const float i18 = v[99];
      v[81] = fmaf(170.9296875f, i8, fmaf(72.515625f, i6, fmaf(11.953125f, i4, fmaf(0.59765625f, i2, 0.00390625f * i0))));
      v[82] = fmaf(27.625f, i7, fmaf(14.875f, i5, fmaf(2.125f, i3, 0.0625f * i1)));
      v[83] = fmaf(-7.8203125f, i8, fmaf(4.265625f, i6, fmaf(3.203125f, i4, fmaf(0.34765625f, i2, 0.00390625f * i0))));
      v[84] = fmaf(-3.65625f, i7, fmaf(0.65625f, i5, fmaf(0.71875f, i3, 0.046875f * i1)));
      v[85] = fmaf(1.1171875f, i8, fmaf(-1.421875f, i6, fmaf(0.140625f, i4, fmaf(0.16015625f, i2, 0.00390625f * i0))));
      v[86] = fmaf(0.8125f, i7, fmaf(-0.5625f, i5, fmaf(0.0625f, i3, 0.03125f * i1)));
      v[87] = fmaf(-0.2578125f, i8, fmaf(0.453125f, i6, fmaf(-0.234375f, i4, fmaf(0.03515625f, i2, 0.00390625f * i0))));
      v[88] = fmaf(-0.21875f, i7, fmaf(0.21875f, i5, fmaf(-0.09375f, i3, 0.015625f * i1)));
      v[89] = fmaf(0.0546875f, i8, fmaf(-0.109375f, i6, fmaf(0.078125f, i4, fmaf(-0.02734375f, i2, 0.00390625f * i0))));
      v[90] = fmaf(0.001953125f, i18, fmaf(-0.017578125f, i16, fmaf(0.0703125f, i14, fmaf(-0.1640625f, i12, 0.24609375f * i10))));
      v[91] = fmaf(0.0078125f, i17, fmaf(-0.0625f, i15, fmaf(0.21875f, i13, fmaf(-0.4375f, i11, 0.546875f * i9))));
      v[92] = fmaf(0.00390625f, i18, fmaf(-0.00390625f, i16, fmaf(-0.078125f, i14, fmaf(0.328125f, i12, -0.6015625f * i10))));
      v[93] = fmaf(0.0234375f, i17, fmaf(-0.0625f, i15, fmaf(-0.09375f, i13, fmaf(0.5625f, i11, -0.859375f * i9))));
      v[94] = fmaf(0.00390625f, i18, fmaf(0.08984375f, i16, fmaf(-0.234375f, i14, fmaf(-0.203125f, i12, 1.1171875f * i10))));
      v[95] = fmaf(0.0390625f, i17, fmaf(0.3125f, i15, fmaf(-0.65625f, i13, fmaf(-0.8125f, i11, 2.234375f * i9))));
      v[96] = fmaf(0.00390625f, i18, fmaf(0.24609375f, i16, fmaf(1.171875f, i14, fmaf(-1.421875f, i12, -3.3515625f * i10))));
      v[97] = fmaf(0.0546875f, i17, fmaf(1.3125f, i15, fmaf(5.03125f, i13, fmaf(-0.8125f, i11, -11.171875f * i9))));
      v[98] = fmaf(0.00390625f, i18, fmaf(0.46484375f, i16, fmaf(6.640625f, i14, fmaf(24.171875f, i12, 18.9921875f * i10))));
      v[99] = fmaf(0.0703125f, i17, fmaf(3.1875f, i15, fmaf(33.46875f, i13, fmaf(124.3125f, i11, 189.921875f * i9))));
    }
    {
      const float i0 = v[100]; const float i1 = v[101]; const float i2 = v[102]; const float i3 = v[103]; const float i4 = v[104]; const float i5 = v[105]; const float i6 = v[106]; const float i7 = v[107]; const float i8 = v[108]; const float i9 = v[109]; const float i10 = v[110]; const float i11 = v[111]; const float i12 = v[112]; const float i13 = v[113]; const float i14 = v[114]; const float i15 = v[115]; const float i16 = v[116]; const float i17 = v[117]; const float i18 = v[118]; const float i19 = v[119]; const float i20 = v[120];
      v[100] = fmaf(328.046875f, i9, fmaf(151.40625f, i7, fmaf(30.28125f, i5, fmaf(2.2265625f, i3, 0.0390625f * i1))));
      v[101] = fmaf(49.20703125f, i8, fmaf(30.28125f, i6, fmaf(5.677734375f, i4, fmaf(0.296875f, i2, 0.001953125f * i0))));
      v[102] = fmaf(-13.8125f, i9, fmaf(6.375f, i7, fmaf(6.375f, i5, fmaf(1.03125f, i3, 0.03125f * i1))));
      v[103] = fmaf(-6.04296875f, i8, fmaf(0.53125f, i6, fmaf(1.427734375f, i4, fmaf(0.171875f, i2, 0.001953125f * i0))));
      v[104] = fmaf(1.828125f, i9, fmaf(-2.15625f, i7, fmaf(-0.03125f, i5, fmaf(0.3359375f, i3, 0.0234375f * i1))));
      v[105] = fmaf(1.26953125f, i8, fmaf(-0.78125f, i6, fmaf(-0.009765625f, i4, fmaf(0.078125f, i2, 0.001953125f * i0))));
      v[106] = fmaf(-0.40625f, i9, fmaf(0.6875f, i7, fmaf(-0.3125f, i5, fmaf(0.015625f, i3, 0.015625f * i1))));
      v[107] = fmaf(-0.35546875f, i8, fmaf(0.34375f, i6, fmaf(-0.134765625f, i4, fmaf(0.015625f, i2, 0.001953125f * i0))));
      v[108] = fmaf(0.109375f, i9, fmaf(-0.21875f, i7, fmaf(0.15625f, i5, fmaf(-0.0546875f, i3, 0.0078125f * i1))));
      v[109] = fmaf(0.08203125f, i8, fmaf(-0.09375f, i6, fmaf(0.052734375f, i4, fmaf(-0.015625f, i2, 0.001953125f * i0))));
      v[110] = fmaf(0.0009765625f, i20, fmaf(-0.009765625f, i18, fmaf(0.0439453125f, i16, fmaf(-0.1171875f, i14, fmaf(0.205078125f, i12, -0.24609375f * i10)))));
      v[111] = fmaf(0.00390625f, i19, fmaf(-0.03515625f, i17, fmaf(0.140625f, i15, fmaf(-0.328125f, i13, 0.4921875f * i11))));
      v[112] = fmaf(0.001953125f, i20, fmaf(-0.00390625f, i18, fmaf(-0.037109375f, i16, fmaf(0.203125f, i14, fmaf(-0.46484375f, i12, 0.6015625f * i10)))));
      v[113] = fmaf(0.01171875f, i19, fmaf(-0.04296875f, i17, fmaf(-0.015625f, i15, fmaf(0.328125f, i13, -0.7109375f * i11))));
      v[114] = fmaf(0.001953125f, i20, fmaf(0.04296875f, i18, fmaf(-0.162109375f, i16, fmaf(0.015625f, i14, fmaf(0.66015625f, i12, -1.1171875f * i10)))));
      v[115] = fmaf(0.01953125f, i19, fmaf(0.13671875f, i17, fmaf(-0.484375f, i15, fmaf(-0.078125f, i13, 1.5234375f * i11))));
      v[116] = fmaf(0.001953125f, i20, fmaf(0.12109375f, i18, fmaf(0.462890625f, i16, fmaf(-1.296875f, i14, fmaf(-0.96484375f, i12, 3.3515625f * i10)))));
      v[117] = fmaf(0.02734375f, i19, fmaf(0.62890625f, i17, fmaf(1.859375f, i15, fmaf(-2.921875f, i13, -5.1796875f * i11))));
      v[118] = fmaf(0.001953125f, i20, fmaf(0.23046875f, i18, fmaf(3.087890625f, i16, fmaf(8.765625f, i14, fmaf(-2.58984375f, i12, -18.9921875f * i10)))));
      v[119] = fmaf(0.03515625f, i19, fmaf(1.55859375f, i17, fmaf(15.140625f, i15, fmaf(45.421875f, i13, 32.8046875f * i11))));
      v[120] = fmaf(0.001953125f, i20, fmaf(0.37109375f, i18, fmaf(9.462890625f, i16, fmaf(75.703125f, i14, fmaf(246.03515625f, i12, 360.8515625f * i10)))));
    }
  }
};
template <int L, bool TR> struct BDeg;
template <> struct BDeg<0, false> {
  static __device__ __forceinline__ void apply(float* v) {
    (void)v;
  }
};
template <> struct BDeg<0, true> {
  static __device__ __forceinline__ void apply(float* v) {
    (void)v;
  }
};
template <> struct BDeg<1, false> {
  static __device__ __forceinline__ void apply(float* v) {
    const float i0 = v[1]; const float i1 = v[2]; const float i2 = v[3];
    v[1] = 1.0f * i0;
    v[2] = 2.0f * i2;
    v[3] = 0.5f * i1;
  }
};
template <> struct BDeg<1, true> {
  static __device__ __forceinline__ void apply(float* v) {
    const float i0 = v[1]; const float i1 = v[2]; const float i2 = v[3];
    v[1] = 1.0f * i0;
    v[2] = 0.5f * i2;
    v[3] = 2.0f * i1;
  }
};
template <> struct BDeg<2, false> {
  static __device__ __forceinline__ void apply(float* v) {
    const float i0 = v[4]; const float i1 = v[5]; const float i2 = v[6]; const float i3 = v[7]; const float i4 = v[8];
    v[4] = 0.5f * i1;
    v[5] = 2.0f * i0;
    v[6] = fmaf(3.0f, i4, -0.5f * i2);
    v[7] = 1.0f * i3;
    v[8] = fmaf(0.5f, i4, 0.25f * i2);
  }
};
template <> struct BDeg<2, true> {
  static __device__ __forceinline__ void apply(float* v) {
    const float i0 = v[4]; const float i1 = v[5]; const float i2 = v[6]; const float i3 = v[7]; const float i4 = v[8];
    v[4] = 2.0f * i1;
    v[5] = 0.5f * i0;
    v[6] = fmaf(0.25f, i4, -0.5f * i2);
    v[7] = 1.0f * i3;
    v[8] = fmaf(0.5f, i4, 3.0f * i2);
  }
};
template <> struct BDeg<3, false> {
  static __device__ __forceinline__ void apply(float* v) {
    const float i0 = v[9]; const float i1 = v[10]; const float i2 = v[11]; const float i3 = v[12]; const float i4 = v[13]; const float i5 = v[14]; const float i6 = v[15];
    v[9] = fmaf(0.25f, i2, 0.25f * i0);
    v[10] = 1.0f * i1;
    v[11] = fmaf(-0.25f, i2, 3.75f * i0);
    v[12] = fmaf(5.0f, i6, -1.0f * i4);
    v[13] = fmaf(1.25f, i5, -0.375f * i3);
    v[14] = fmaf(1.5f, i6, 0.5f * i4);
    v[15] = fmaf(0.25f, i5, 0.125f * i3);
  }
};
template <> struct BDeg<3, true> {
  static __device__ __forceinline__ void apply(float* v) {
    const float i0 = v[9]; const float i1 = v[10]; const float i2 = v[11]; const float i3 = v[12]; const float i4 = v[13]; const float i5 = v[14]; const float i6 = v[15];
    v[9] = fmaf(3.75f, i2, 0.25f * i0);
    v[10] = 1.0f * i1;
    v[11] = fmaf(-0.25f, i2, 0.25f * i0);
    v[12] = fmaf(0.125f, i6, -0.375f * i4);
    v[13] = fmaf(0.5f, i5, -1.0f * i3);
    v[14] = fmaf(0.25f, i6, 1.25f * i4);
    v[15] = fmaf(1.5f, i5, 5.0f * i3);
  }
};
template <> struct BDeg<4, false> {
  static __device__ __forceinline__ void apply(float* v) {
    const float i0 = v[16]; const float i1 = v[17]; const float i2 = v[18]; const float i3 = v[19]; const float i4 = v[20]; const float i5 = v[21]; const float i6 = v[22]; const float i7 = v[23]; const float i8 = v[24];
    v[16] = fmaf(0.125f, i3, 0.125f * i1);
    v[17] = fmaf(0.5f, i2, 1.0f * i0);
    v[18] = fmaf(-0.25f, i3, 1.75f * i1);
    v[19] = fmaf(-0.5f, i2, 7.0f * i0);
    v[20] = fmaf(8.75f, i8, fmaf(-1.25f, i6, 0.375f * i4));
    v[21] = fmaf(1.75f, i7, -0.75f * i5);
    v[22] = fmaf(3.5f, i8, fmaf(0.5f, i6, -0.25f * i4));
    v[23] = fmaf(0.75f, i7, 0.25f * i5);
    v[24] = fmaf(0.125f, i8, fmaf(0.125f, i6, 0.0625f * i4));
  }
};
template <> struct BDeg<4, true> {
  static __device__ __forceinline__ void apply(float* v) {
    const float i0 = v[16]; const float i1 = v[17]; const float i2 = v[18]; const float i3 = v[19]; const float i4 = v[20]; const float i5 = v[21]; const float i6 = v[22]; const float i7 = v[23]; const float i8 = v[24];
    v[16] = fmaf(7.0f, i3, 1.0f * i1);
    v[17] = fmaf(1.75f, i2, 0.125f * i0);
    v[18] = fmaf(-0.5f, i3, 0.5f * i1);
    v[19] = fmaf(-0.25f, i2, 0.125f * i0);
    v[20] = fmaf(0.0625f, i8, fmaf(-0.25f, i6, 0.375f * i4));
    v[21] = fmaf(0.25f, i7, -0.75f * i5);
    v[22] = fmaf(0.125f, i8, fmaf(0.5f, i6, -1.25f * i4));
    v[23] = fmaf(0.75f, i7, 1.75f * i5);
    v[24] = fmaf(0.125f, i8, fmaf(3.5f, i6, 8.75f * i4));
  }
};
template <> struct BDeg<5, false> {
  static __device__ __forceinline__ void apply(float* v) {
    const float i0 = v[25]; const float i1 = v[26]; const float i2 = v[27]; const float i3 = v[28]; const float i4 = v[29]; const float i5 = v[30]; const float i6 = v[31]; const float i7 = v[32]; const float i8 = v[33]; const float i9 = v[34]; const float i10 = v[35];
    v[25] = fmaf(0.0625f, i4, fmaf(0.0625f, i2, 0.0625f * i0));
    v[26] = fmaf(0.25f, i3, 0.5f * i1);
    v[27] = fmaf(-0.1875f, i4, fmaf(0.8125f, i2, 2.8125f * i0));
    v[28] = fmaf(-0.5f, i3, 3.0f * i1);
    v[29] = fmaf(0.125f, i4, fmaf(-0.875f, i2, 13.125f * i0));
    v[30] = fmaf(15.75f, i10, fmaf(-1.75f, i8, 0.75f * i6));
    v[31] = fmaf(2.625f, i9, fmaf(-0.875f, i7, 0.3125f * i5));
    v[32] = fmaf(7.5f, i10, fmaf(0.5f, i8, -0.5f * i6));
    v[33] = fmaf(1.6875f, i9, fmaf(0.1875f, i7, -0.15625f * i5));
    v[34] = fmaf(0.625f, i10, fmaf(0.375f, i8, 0.125f * i6));
    v[35] = fmaf(0.0625f, i9, fmaf(0.0625f, i7, 0.03125f * i5));
  }
};
template <> struct BDeg<5, true> {
  static __device__ __forceinline__ void apply(float* v) {
    const float i0 = v[25]; const float i1 = v[26]; const float i2 = v[27]; const float i3 = v[28]; const float i4 = v[29]; const float i5 = v[30]; const float i6 = v[31]; const float i7 = v[32]; const float i8 = v[33]; const float i9 = v[34]; const float i10 = v[35];
    v[25] = fmaf(13.125f, i4, fmaf(2.8125f, i2, 0.0625f * i0));
    v[26] = fmaf(3.0f, i3, 0.5f * i1);
    v[27] = fmaf(-0.875f, i4, fmaf(0.8125f, i2, 0.0625f * i0));
    v[28] = fmaf(-0.5f, i3, 0.25f * i1);
    v[29] = fmaf(0.125f, i4, fmaf(-0.1875f, i2, 0.0625f * i0));
    v[30] = fmaf(0.03125f, i10, fmaf(-0.15625f, i8, 0.3125f * i6));
    v[31] = fmaf(0.125f, i9, fmaf(-0.5f, i7, 0.75f * i5));
    v[32] = fmaf(0.0625f, i10, fmaf(0.1875f, i8, -0.875f * i6));
    v[33] = fmaf(0.375f, i9, fmaf(0.5f, i7, -1.75f * i5));
    v[34] = fmaf(0.0625f, i10, fmaf(1.6875f, i8, 2.625f * i6));
    v[35] = fmaf(0.625f, i9, fmaf(7.5f, i7, 15.75f * i5));
  }
};
template <> struct BDeg<6, false> {
  static __device__ __forceinline__ void apply(float* v) {
    const float i0 = v[36]; const float i1 = v[37]; const float i2 = v[38]; const float i3 = v[39]; const float i4 = v[40]; const float i5 = v[41]; const float i6 = v[42]; const float i7 = v[43]; const float i8 = v[44]; const float i9 = v[45]; const float i10 = v[46]; const float i11 = v[47]; const float i12 = v[48];
    v[36] = fmaf(0.03125f, i5, fmaf(0.03125f, i3, 0.03125f * i1));
    v[37] = fmaf(0.125f, i4, fmaf(0.25f, i2, 0.375f * i0));
    v[38] = fmaf(-0.125f, i5, fmaf(0.375f, i3, 1.375f * i1));
    v[39] = fmaf(-0.375f, i4, fmaf(1.25f, i2, 6.875f * i0));
    v[40] = fmaf(0.15625f, i5, fmaf(-0.84375f, i3, 5.15625f * i1));
    v[41] = fmaf(0.25f, i4, fmaf(-1.5f, i2, 24.75f * i0));
    v[42] = fmaf(28.875f, i12, fmaf(-2.625f, i10, fmaf(0.875f, i8, -0.3125f * i6)));
    v[43] = fmaf(4.125f, i11, fmaf(-1.125f, i9, 0.625f * i7));
    v[44] = fmaf(15.46875f, i12, fmaf(0.46875f, i10, fmaf(-0.53125f, i8, 0.234375f * i6)));
    v[45] = fmaf(3.4375f, i11, fmaf(0.0625f, i9, -0.3125f * i7));
    v[46] = fmaf(2.0625f, i12, fmaf(0.8125f, i10, fmaf(0.0625f, i8, -0.09375f * i6)));
    v[47] = fmaf(0.3125f, i11, fmaf(0.1875f, i9, 0.0625f * i7));
    v[48] = fmaf(0.03125f, i12, fmaf(0.03125f, i10, fmaf(0.03125f, i8, 0.015625f * i6)));
  }
};
template <> struct BDeg<6, true> {
  static __device__ __forceinline__ void apply(float* v) {
    const float i0 = v[36]; const float i1 = v[37]; const float i2 = v[38]; const float i3 = v[39]; const float i4 = v[40]; const float i5 = v[41]; const float i6 = v[42]; const float i7 = v[43]; const float i8 = v[44]; const float i9 = v[45]; const float i10 = v[46]; const float i11 = v[47]; const float i12 = v[48];
    v[36] = fmaf(24.75f, i5, fmaf(6.875f, i3, 0.375f * i1));
    v[37] = fmaf(5.15625f, i4, fmaf(1.375f, i2, 0.03125f * i0));
    v[38] = fmaf(-1.5f, i5, fmaf(1.25f, i3, 0.25f * i1));
    v[39] = fmaf(-0.84375f, i4, fmaf(0.375f, i2, 0.03125f * i0));
    v[40] = fmaf(0.25f, i5, fmaf(-0.375f, i3, 0.125f * i1));
    v[41] = fmaf(0.15625f, i4, fmaf(-0.125f, i2, 0.03125f * i0));
    v[42] = fmaf(0.015625f, i12, fmaf(-0.09375f, i10, fmaf(0.234375f, i8, -0.3125f * i6)));
    v[43] = fmaf(0.0625f, i11, fmaf(-0.3125f, i9, 0.625f * i7));
    v[44] = fmaf(0.03125f, i12, fmaf(0.0625f, i10, fmaf(-0.53125f, i8, 0.875f * i6)));
    v[45] = fmaf(0.1875f, i11, fmaf(0.0625f, i9, -1.125f * i7));
    v[46] = fmaf(0.03125f, i12, fmaf(0.8125f, i10, fmaf(0.46875f, i8, -2.625f * i6)));
    v[47] = fmaf(0.3125f, i11, fmaf(3.4375f, i9, 4.125f * i7));
    v[48] = fmaf(0.03125f, i12, fmaf(2.0625f, i10, fmaf(15.46875f, i8, 28.875f * i6)));
  }
};
template <> struct BDeg<7, false> {
  static __device__ __forceinline__ void apply(float* v) {
    const float i0 = v[49]; const float i1 = v[50]; const float i2 = v[51]; const float i3 = v[52]; const float i4 = v[53]; const float i5 = v[54]; const float i6 = v[55]; const float i7 = v[56]; const float i8 = v[57]; const float i9 = v[58]; const float i10 = v[59]; const float i11 = v[60]; const float i12 = v[61]; const float i13 = v[62]; const float i14 = v[63];
    v[49] = fmaf(0.015625f, i6, fmaf(0.015625f, i4, fmaf(0.015625f, i2, 0.015625f * i0)));
    v[50] = fmaf(0.0625f, i5, fmaf(0.125f, i3, 0.1875f * i1));
    v[51] = fmaf(-0.078125f, i6, fmaf(0.171875f, i4, fmaf(0.671875f, i2, 1.421875f * i0)));
    v[52] = fmaf(-0.25f, i5, fmaf(0.5f, i3, 3.25f * i1));
    v[53] = fmaf(0.140625f, i6, fmaf(-0.609375f, i4, fmaf(1.890625f, i2, 15.640625f * i0)));
    v[54] = fmaf(0.3125f, i5, fmaf(-1.375f, i3, 8.9375f * i1));
    v[55] = fmaf(-0.078125f, i6, fmaf(0.421875f, i4, fmaf(-2.578125f, i2, 46.921875f * i0)));
    v[56] = fmaf(53.625f, i14, fmaf(-4.125f, i12, fmaf(1.125f, i10, -0.625f * i8)));
    v[57] = fmaf(6.703125f, i13, fmaf(-1.546875f, i11, fmaf(0.703125f, i9, -0.2734375f * i7)));
    v[58] = fmaf(31.28125f, i14, fmaf(0.34375f, i12, fmaf(-0.59375f, i10, 0.46875f * i8)));
    v[59] = fmaf(6.703125f, i13, fmaf(-0.171875f, i11, fmaf(-0.296875f, i9, 0.1640625f * i7)));
    v[60] = fmaf(5.6875f, i14, fmaf(1.5625f, i12, fmaf(-0.0625f, i10, -0.1875f * i8)));
    v[61] = fmaf(1.015625f, i13, fmaf(0.390625f, i11, fmaf(0.015625f, i9, -0.0546875f * i7)));
    v[62] = fmaf(0.21875f, i14, fmaf(0.15625f, i12, fmaf(0.09375f, i10, 0.03125f * i8)));
    v[63] = fmaf(0.015625f, i13, fmaf(0.015625f, i11, fmaf(0.015625f, i9, 0.0078125f * i7)));
  }
};
template <> struct BDeg<7, true> {
  static __device__ __forceinline__ void apply(float* v) {
    const float i0 = v[49]; const float i1 = v[50]; const float i2 = v[51]; const float i3 = v[52]; const float i4 = v[53]; const float i5 = v[54]; const float i6 = v[55]; const float i7 = v[56]; const float i8 = v[57]; const float i9 = v[58]; const float i10 = v[59]; const float i11 = v[60]; const float i12 = v[61]; const float i13 = v[62]; const float i14 = v[63];
    v[49] = fmaf(46.921875f, i6, fmaf(15.640625f, i4, fmaf(1.421875f, i2, 0.015625f * i0)));
    v[50] = fmaf(8.9375f, i5, fmaf(3.25f, i3, 0.1875f * i1));
    v[51] = fmaf(-2.578125f, i6, fmaf(1.890625f, i4, fmaf(0.671875f, i2, 0.015625f * i0)));
    v[52] = fmaf(-1.375f, i5, fmaf(0.5f, i3, 0.125f * i1));
    v[53] = fmaf(0.421875f, i6, fmaf(-0.609375f, i4, fmaf(0.171875f, i2, 0.015625f * i0)));
    v[54] = fmaf(0.3125f, i5, fmaf(-0.25f, i3, 0.0625f * i1));
    v[55] = fmaf(-0.078125f, i6, fmaf(0.140625f, i4, fmaf(-0.078125f, i2, 0.015625f * i0)));
    v[56] = fmaf(0.0078125f, i14, fmaf(-0.0546875f, i12, fmaf(0.1640625f, i10, -0.2734375f * i8)));
    v[57] = fmaf(0.03125f, i13, fmaf(-0.1875f, i11, fmaf(0.46875f, i9, -0.625f * i7)));
    v[58] = fmaf(0.015625f, i14, fmaf(0.015625f, i12, fmaf(-0.296875f, i10, 0.703125f * i8)));
    v[59] = fmaf(0.09375f, i13, fmaf(-0.0625f, i11, fmaf(-0.59375f, i9, 1.125f * i7)));
    v[60] = fmaf(0.015625f, i14, fmaf(0.390625f, i12, fmaf(-0.171875f, i10, -1.546875f * i8)));
    v[61] = fmaf(0.15625f, i13, fmaf(1.5625f, i11, fmaf(0.34375f, i9, -4.125f * i7)));
    v[62] = fmaf(0.015625f, i14, fmaf(1.015625f, i12, fmaf(6.703125f, i10, 6.703125f * i8)));
    v[63] = fmaf(0.21875f, i13, fmaf(5.6875f, i11, fmaf(31.28125f, i9, 53.625f * i7)));
  }
};
template <> struct BDeg<8, false> {
  static __device__ __forceinline__ void apply(float* v) {
    const float i0 = v[64]; const float i1 = v[65]; const float i2 = v[66]; const float i3 = v[67]; const float i4 = v[68]; const float i5 = v[69]; const float i6 = v[70]; const float i7 = v[71]; const float i8 = v[72]; const float i9 = v[73]; const float i10 = v[74]; const float i11 = v[75]; const float i12 = v[76]; const float i13 = v[77]; const float i14 = v[78]; const float i15 = v[79]; const float i16 = v[80];
    v[64] = fmaf(0.0078125f, i7, fmaf(0.0078125f, i5, fmaf(0.0078125f, i3, 0.0078125f * i1)));
    v[65] = fmaf(0.03125f, i6, fmaf(0.0625f, i4, fmaf(0.09375f, i2, 0.125f * i0)));
    v[66] = fmaf(-0.046875f, i7, fmaf(0.078125f, i5, fmaf(0.328125f, i3, 0.703125f * i1)));
    v[67] = fmaf(-0.15625f, i6, fmaf(0.1875f, i4, fmaf(1.53125f, i2, 4.375f * i0)));
    v[68] = fmaf(0.109375f, i7, fmaf(-0.390625f, i5, fmaf(0.609375f, i3, 7.109375f * i1)));
    v[69] = fmaf(0.28125f, i6, fmaf(-0.9375f, i4, fmaf(2.84375f, i2, 34.125f * i0)));
    v[70] = fmaf(-0.109375f, i7, fmaf(0.515625f, i5, fmaf(-2.234375f, i3, 15.640625f * i1)));
    v[71] = fmaf(-0.15625f, i6, fmaf(0.6875f, i4, fmaf(-4.46875f, i2, 89.375f * i0)));
    v[72] = fmaf(100.546875f, i16, fmaf(-6.703125f, i14, fmaf(1.546875f, i12, fmaf(-0.703125f, i10, 0.2734375f * i8))));
    v[73] = fmaf(11.171875f, i15, fmaf(-2.234375f, i13, fmaf(0.859375f, i11, -0.546875f * i9)));
    v[74] = fmaf(62.5625f, i16, fmaf(-0.6875f, i12, fmaf(0.5f, i10, -0.21875f * i8)));
    v[75] = fmaf(12.796875f, i15, fmaf(-0.609375f, i13, fmaf(-0.265625f, i11, 0.328125f * i9)));
    v[76] = fmaf(14.21875f, i16, fmaf(2.84375f, i14, fmaf(-0.28125f, i12, fmaf(-0.15625f, i10, 0.109375f * i8))));
    v[77] = fmaf(2.734375f, i15, fmaf(0.703125f, i13, fmaf(-0.078125f, i11, -0.109375f * i9)));
    v[78] = fmaf(0.9375f, i16, fmaf(0.5f, i14, fmaf(0.1875f, i12, -0.03125f * i8)));
    v[79] = fmaf(0.109375f, i15, fmaf(0.078125f, i13, fmaf(0.046875f, i11, 0.015625f * i9)));
    v[80] = fmaf(0.0078125f, i16, fmaf(0.0078125f, i14, fmaf(0.0078125f, i12, fmaf(0.0078125f, i10, 0.00390625f * i8))));
  }
};
template <> struct BDeg<8, true> {
  static __device__ __forceinline__ void apply(float* v) {
    const float i0 = v[64]; const float i1 = v[65]; const float i2 = v[66]; const float i3 = v[67]; const float i4 = v[68]; const float i5 = v[69]; const float i6 = v[70]; const float i7 = v[71]; const float i8 = v[72]; const float i9 = v[73]; const float i10 = v[74]; const float i11 = v[75]; const float i12 = v[76]; const float i13 = v[77]; const float i14 = v[78]; const float i15 = v[79]; const float i16 = v[80];
    v[64] = fmaf(89.375f, i7, fmaf(34.125f, i5, fmaf(4.375f, i3, 0.125f * i1)));
    v[65] = fmaf(15.640625f, i6, fmaf(7.109375f, i4, fmaf(0.703125f, i2, 0.0078125f * i0)));
    v[66] = fmaf(-4.46875f, i7, fmaf(2.84375f, i5, fmaf(1.53125f, i3, 0.09375f * i1)));
    v[67] = fmaf(-2.234375f, i6, fmaf(0.609375f, i4, fmaf(0.328125f, i2, 0.0078125f * i0)));
    v[68] = fmaf(0.6875f, i7, fmaf(-0.9375f, i5, fmaf(0.1875f, i3, 0.0625f * i1)));
    v[69] = fmaf(0.515625f, i6, fmaf(-0.390625f, i4, fmaf(0.078125f, i2, 0.0078125f * i0)));
    v[70] = fmaf(-0.15625f, i7, fmaf(0.28125f, i5, fmaf(-0.15625f, i3, 0.03125f * i1)));
    v[71] = fmaf(-0.109375f, i6, fmaf(0.109375f, i4, fmaf(-0.046875f, i2, 0.0078125f * i0)));
    v[72] = fmaf(0.00390625f, i16, fmaf(-0.03125f, i14, fmaf(0.109375f, i12, fmaf(-0.21875f, i10, 0.2734375f * i8))));
    v[73] = fmaf(0.015625f, i15, fmaf(-0.109375f, i13, fmaf(0.328125f, i11, -0.546875f * i9)));
    v[74] = fmaf(0.0078125f, i16, fmaf(-0.15625f, i12, fmaf(0.5f, i10, -0.703125f * i8)));
    v[75] = fmaf(0.046875f, i15, fmaf(-0.078125f, i13, fmaf(-0.265625f, i11, 0.859375f * i9)));
    v[76] = fmaf(0.0078125f, i16, fmaf(0.1875f, i14, fmaf(-0.28125f, i12, fmaf(-0.6875f, i10, 1.546875f * i8))));
    v[77] = fmaf(0.078125f, i15, fmaf(0.703125f, i13, fmaf(-0.609375f, i11, -2.234375f * i9)));
    v[78] = fmaf(0.0078125f, i16, fmaf(0.5f, i14, fmaf(2.84375f, i12, -6.703125f * i8)));
    v[79] = fmaf(0.109375f, i15, fmaf(2.734375f, i13, fmaf(12.796875f, i11, 11.171875f * i9)));
    v[80] = fmaf(0.0078125f, i16, fmaf(0.9375f, i14, fmaf(14.21875f, i12, fmaf(62.5625f, i10, 100.546875f * i8))));
  }
};
template <> struct BDeg<9, false> {
  static __device__ __forceinline__ void apply(float* v) {
    const float i0 = v[81]; const float i1 = v[82]; const float i2 = v[83]; const float i3 = v[84]; const float i4 = v[85]; const float i5 = v[86]; const float i6 = v[87]; const float i7 = v[88]; const float i8 = v[89]; const float i9 = v[90]; const float i10 = v[91]; const float i11 = v[92]; const float i12 = v[93]; const float i13 = v[94]; const float i14 = v[95]; const float i15 = v[96]; const float i16 = v[97]; const float i17 = v[98]; const float i18 = v[99];
    v[81] = fmaf(0.00390625f, i8, fmaf(0.00390625f, i6, fmaf(0.00390625f, i4, fmaf(0.00390625f, i2, 0.00390625f * i0))));
    v[82] = fmaf(0.015625f, i7, fmaf(0.03125f, i5, fmaf(0.046875f, i3, 0.0625f * i1)));
    v[83] = fmaf(-0.02734375f, i8, fmaf(0.03515625f, i6, fmaf(0.16015625f, i4, fmaf(0.34765625f, i2, 0.59765625f * i0))));
    v[84] = fmaf(-0.09375f, i7, fmaf(0.0625f, i5, fmaf(0.71875f, i3, 2.125f * i1)));
    v[85] = fmaf(0.078125f, i8, fmaf(-0.234375f, i6, fmaf(0.140625f, i4, fmaf(3.203125f, i2, 11.953125f * i0))));
    v[86] = fmaf(0.21875f, i7, fmaf(-0.5625f, i5, fmaf(0.65625f, i3, 14.875f * i1)));
    v[87] = fmaf(-0.109375f, i8, fmaf(0.453125f, i6, fmaf(-1.421875f, i4, fmaf(4.265625f, i2, 72.515625f * i0))));
    v[88] = fmaf(-0.21875f, i7, fmaf(0.8125f, i5, fmaf(-3.65625f, i3, 27.625f * i1)));
    v[89] = fmaf(0.0546875f, i8, fmaf(-0.2578125f, i6, fmaf(1.1171875f, i4, fmaf(-7.8203125f, i2, 170.9296875f * i0))));
    v[90] = fmaf(189.921875f, i18, fmaf(-11.171875f, i16, fmaf(2.234375f, i14, fmaf(-0.859375f, i12, 0.546875f * i10))));
    v[91] = fmaf(18.9921875f, i17, fmaf(-3.3515625f, i15, fmaf(1.1171875f, i13, fmaf(-0.6015625f, i11, 0.24609375f * i9))));
    v[92] = fmaf(124.3125f, i18, fmaf(-0.8125f, i16, fmaf(-0.8125f, i14, fmaf(0.5625f, i12, -0.4375f * i10))));
    v[93] = fmaf(24.171875f, i17, fmaf(-1.421875f, i15, fmaf(-0.203125f, i13, fmaf(0.328125f, i11, -0.1640625f * i9))));
    v[94] = fmaf(33.46875f, i18, fmaf(5.03125f, i16, fmaf(-0.65625f, i14, fmaf(-0.09375f, i12, 0.21875f * i10))));
    v[95] = fmaf(6.640625f, i17, fmaf(1.171875f, i15, fmaf(-0.234375f, i13, fmaf(-0.078125f, i11, 0.0703125f * i9))));
    v[96] = fmaf(3.1875f, i18, fmaf(1.3125f, i16, fmaf(0.3125f, i14, fmaf(-0.0625f, i12, -0.0625f * i10))));
    v[97] = fmaf(0.46484375f, i17, fmaf(0.24609375f, i15, fmaf(0.08984375f, i13, fmaf(-0.00390625f, i11, -0.017578125f * i9))));
    v[98] = fmaf(0.0703125f, i18, fmaf(0.0546875f, i16, fmaf(0.0390625f, i14, fmaf(0.0234375f, i12, 0.0078125f * i10))));
    v[99] = fmaf(0.00390625f, i17, fmaf(0.00390625f, i15, fmaf(0.00390625f, i13, fmaf(0.00390625f, i11, 0.001953125f * i9))));
  }
};
template <> struct BDeg<9, true> {
  static __device__ __forceinline__ void apply(float* v) {
    const float i0 = v[81]; const float i1 = v[82]; const float i2 = v[83]; const float i3 = v[84]; const float i4 = v[85]; const float i5 = v[86]; const float i6 = v[87]; const float i7 = v[88]; const float i8 = v[89]; const float i9 = v[90]; const float i10 = v[91]; const float i11 = v[92]; const float i12 = v[93]; const float i13 = v[94]; const float i14 = v[95]; const float i15 = v[96]; const float i16 = v[97]; const float i17 = v[98]; const float i18 = v[99];
    v[81] = fmaf(170.9296875f, i8, fmaf(72.515625f, i6, fmaf(11.953125f, i4, fmaf(0.59765625f, i2, 0.00390625f * i0))));
    v[82] = fmaf(27.625f, i7, fmaf(14.875f, i5, fmaf(2.125f, i3, 0.0625f * i1)));
    v[83] = fmaf(-7.8203125f, i8, fmaf(4.265625f, i6, fmaf(3.203125f, i4, fmaf(0.34765625f, i2, 0.00390625f * i0))));
    v[84] = fmaf(-3.65625f, i7, fmaf(0.65625f, i5, fmaf(0.71875f, i3, 0.046875f * i1)));
    v[85] = fmaf(1.1171875f, i8, fmaf(-1.421875f, i6, fmaf(0.140625f, i4, fmaf(0.16015625f, i2, 0.00390625f * i0))));
    v[86] = fmaf(0.8125f, i7, fmaf(-0.5625f, i5, fmaf(0.0625f, i3, 0.03125f * i1)));
    v[87] = fmaf(-0.2578125f, i8, fmaf(0.453125f, i6, fmaf(-0.234375f, i4, fmaf(0.03515625f, i2, 0.00390625f * i0))));
    v[88] = fmaf(-0.21875f, i7, fmaf(0.21875f, i5, fmaf(-0.09375f, i3, 0.015625f * i1)));
    v[89] = fmaf(0.0546875f, i8, fmaf(-0.109375f, i6, fmaf(0.078125f, i4, fmaf(-0.02734375f, i2, 0.00390625f * i0))));
    v[90] = fmaf(0.001953125f, i18, fmaf(-0.017578125f, i16, fmaf(0.0703125f, i14, fmaf(-0.1640625f, i12, 0.24609375f * i10))));
    v[91] = fmaf(0.0078125f, i17, fmaf(-0.0625f, i15, fmaf(0.21875f, i13, fmaf(-0.4375f, i11, 0.546875f * i9))));
    v[92] = fmaf(0.00390625f, i18, fmaf(-0.00390625f, i16, fmaf(-0.078125f, i14, fmaf(0.328125f, i12, -0.6015625f * i10))));
    v[93] = fmaf(0.0234375f, i17, fmaf(-0.0625f, i15, fmaf(-0.09375f, i13, fmaf(0.5625f, i11, -0.859375f * i9))));
    v[94] = fmaf(0.00390625f, i18, fmaf(0.08984375f, i16, fmaf(-0.234375f, i14, fmaf(-0.203125f, i12, 1.1171875f * i10))));
    v[95] = fmaf(0.0390625f, i17, fmaf(0.3125f, i15, fmaf(-0.65625f, i13, fmaf(-0.8125f, i11, 2.234375f * i9))));
    v[96] = fmaf(0.00390625f, i18, fmaf(0.24609375f, i16, fmaf(1.171875f, i14, fmaf(-1.421875f, i12, -3.3515625f * i10))));
    v[97] = fmaf(0.0546875f, i17, fmaf(1.3125f, i15, fmaf(5.03125f, i13, fmaf(-0.8125f, i11, -11.171875f * i9))));
    v[98] = fmaf(0.00390625f, i18, fmaf(0.46484375f, i16, fmaf(6.640625f, i14, fmaf(24.171875f, i12, 18.9921875f * i10))));
    v[99] = fmaf(0.0703125f, i17, fmaf(3.1875f, i15, fmaf(33.46875f, i13, fmaf(124.3125f, i11, 189.921875f * i9))));
  }
};
template <> struct BDeg<10, false> {
  static __device__ __forceinline__ void apply(float* v) {
    const float i0 = v[100]; const float i1 = v[101]; const float i2 = v[102]; const float i3 = v[103]; const float i4 = v[104]; const float i5 = v[105]; const float i6 = v[106]; const float i7 = v[107]; const float i8 = v[108]; const float i9 = v[109]; const float i10 = v[110]; const float i11 = v[111]; const float i12 = v[112]; const float i13 = v[113]; const float i14 = v[114]; const float i15 = v[115]; const float i16 = v[116]; const float i17 = v[117]; const float i18 = v[118]; const float i19 = v[119]; const float i20 = v[120];
    v[100] = fmaf(0.001953125f, i9, fmaf(0.001953125f, i7, fmaf(0.001953125f, i5, fmaf(0.001953125f, i3, 0.001953125f * i1))));
    v[101] = fmaf(0.0078125f, i8, fmaf(0.015625f, i6, fmaf(0.0234375f, i4, fmaf(0.03125f, i2, 0.0390625f * i0))));
    v[102] = fmaf(-0.015625f, i9, fmaf(0.015625f, i7, fmaf(0.078125f, i5, fmaf(0.171875f, i3, 0.296875f * i1))));
    v[103] = fmaf(-0.0546875f, i8, fmaf(0.015625f, i6, fmaf(0.3359375f, i4, fmaf(1.03125f, i2, 2.2265625f * i0))));
    v[104] = fmaf(0.052734375f, i9, fmaf(-0.134765625f, i7, fmaf(-0.009765625f, i5, fmaf(1.427734375f, i3, 5.677734375f * i1))));
    v[105] = fmaf(0.15625f, i8, fmaf(-0.3125f, i6, fmaf(-0.03125f, i4, fmaf(6.375f, i2, 30.28125f * i0))));
    v[106] = fmaf(-0.09375f, i9, fmaf(0.34375f, i7, fmaf(-0.78125f, i5, fmaf(0.53125f, i3, 30.28125f * i1))));
    v[107] = fmaf(-0.21875f, i8, fmaf(0.6875f, i6, fmaf(-2.15625f, i4, fmaf(6.375f, i2, 151.40625f * i0))));
    v[108] = fmaf(0.08203125f, i9, fmaf(-0.35546875f, i7, fmaf(1.26953125f, i5, fmaf(-6.04296875f, i3, 49.20703125f * i1))));
    v[109] = fmaf(0.109375f, i8, fmaf(-0.40625f, i6, fmaf(1.828125f, i4, fmaf(-13.8125f, i2, 328.046875f * i0))));
    v[110] = fmaf(360.8515625f, i20, fmaf(-18.9921875f, i18, fmaf(3.3515625f, i16, fmaf(-1.1171875f, i14, fmaf(0.6015625f, i12, -0.24609375f * i10)))));
    v[111] = fmaf(32.8046875f, i19, fmaf(-5.1796875f, i17, fmaf(1.5234375f, i15, fmaf(-0.7109375f, i13, 0.4921875f * i11))));
    v[112] = fmaf(246.03515625f, i20, fmaf(-2.58984375f, i18, fmaf(-0.96484375f, i16, fmaf(0.66015625f, i14, fmaf(-0.46484375f, i12, 0.205078125f * i10)))));
    v[113] = fmaf(45.421875f, i19, fmaf(-2.921875f, i17, fmaf(-0.078125f, i15, fmaf(0.328125f, i13, -0.328125f * i11))));
    v[114] = fmaf(75.703125f, i20, fmaf(8.765625f, i18, fmaf(-1.296875f, i16, fmaf(0.015625f, i14, fmaf(0.203125f, i12, -0.1171875f * i10)))));
    v[115] = fmaf(15.140625f, i19, fmaf(1.859375f, i17, fmaf(-0.484375f, i15, fmaf(-0.015625f, i13, 0.140625f * i11))));
    v[116] = fmaf(9.462890625f, i20, fmaf(3.087890625f, i18, fmaf(0.462890625f, i16, fmaf(-0.162109375f, i14, fmaf(-0.037109375f, i12, 0.0439453125f * i10)))));
    v[117] = fmaf(1.55859375f, i19, fmaf(0.62890625f, i17, fmaf(0.13671875f, i15, fmaf(-0.04296875f, i13, -0.03515625f * i11))));
    v[118] = fmaf(0.37109375f, i20, fmaf(0.23046875f, i18, fmaf(0.12109375f, i16, fmaf(0.04296875f, i14, fmaf(-0.00390625f, i12, -0.009765625f * i10)))));
    v[119] = fmaf(0.03515625f, i19, fmaf(0.02734375f, i17, fmaf(0.01953125f, i15, fmaf(0.01171875f, i13, 0.00390625f * i11))));
    v[120] = fmaf(0.001953125f, i20, fmaf(0.001953125f, i18, fmaf(0.001953125f, i16, fmaf(0.001953125f, i14, fmaf(0.001953125f, i12, 0.0009765625f * i10)))));
  }
};
template <> struct BDeg<10, true> {
  static __device__ __forceinline__ void apply(float* v) {
    const float i0 = v[100]; const float i1 = v[101]; const float i2 = v[102]; const float i3 = v[103]; const float i4 = v[104]; const float i5 = v[105]; const float i6 = v[106]; const float i7 = v[107]; const float i8 = v[108]; const float i9 = v[109]; const float i10 = v[110]; const float i11 = v[111]; const float i12 = v[112]; const float i13 = v[113]; const float i14 = v[114]; const float i15 = v[115]; const float i16 = v[116]; const float i17 = v[117]; const float i18 = v[118]; const float i19 = v[119]; const float i20 = v[120];
    v[100] = fmaf(328.046875f, i9, fmaf(151.40625f, i7, fmaf(30.28125f, i5, fmaf(2.2265625f, i3, 0.0390625f * i1))));
    v[101] = fmaf(49.20703125f, i8, fmaf(30.28125f, i6, fmaf(5.677734375f, i4, fmaf(0.296875f, i2, 0.001953125f * i0))));
    v[102] = fmaf(-13.8125f, i9, fmaf(6.375f, i7, fmaf(6.375f, i5, fmaf(1.03125f, i3, 0.03125f * i1))));
    v[103] = fmaf(-6.04296875f, i8, fmaf(0.53125f, i6, fmaf(1.427734375f, i4, fmaf(0.171875f, i2, 0.001953125f * i0))));
    v[104] = fmaf(1.828125f, i9, fmaf(-2.15625f, i7, fmaf(-0.03125f, i5, fmaf(0.3359375f, i3, 0.0234375f * i1))));
    v[105] = fmaf(1.26953125f, i8, fmaf(-0.78125f, i6, fmaf(-0.009765625f, i4, fmaf(0.078125f, i2, 0.001953125f * i0))));
    v[106] = fmaf(-0.40625f, i9, fmaf(0.6875f, i7, fmaf(-0.3125f, i5, fmaf(0.015625f, i3, 0.015625f * i1))));
    v[107] = fmaf(-0.35546875f, i8, fmaf(0.34375f, i6, fmaf(-0.134765625f, i4, fmaf(0.015625f, i2, 0.001953125f * i0))));
    v[108] = fmaf(0.109375f, i9, fmaf(-0.21875f, i7, fmaf(0.15625f, i5, fmaf(-0.0546875f, i3, 0.0078125f * i1))));
    v[109] = fmaf(0.08203125f, i8, fmaf(-0.09375f, i6, fmaf(0.052734375f, i4, fmaf(-0.015625f, i2, 0.001953125f * i0))));
    v[110] = fmaf(0.0009765625f, i20, fmaf(-0.009765625f, i18, fmaf(0.0439453125f, i16, fmaf(-0.1171875f, i14, fmaf(0.205078125f, i12, -0.24609375f * i10)))));
    v[111] = fmaf(0.00390625f, i19, fmaf(-0.03515625f, i17, fmaf(0.140625f, i15, fmaf(-0.328125f, i13, 0.4921875f * i11))));
    v[112] = fmaf(0.001953125f, i20, fmaf(-0.00390625f, i18, fmaf(-0.037109375f, i16, fmaf(0.203125f, i14, fmaf(-0.46484375f, i12, 0.6015625f * i10)))));
    v[113] = fmaf(0.01171875f, i19, fmaf(-0.04296875f, i17, fmaf(-0.015625f, i15, fmaf(0.328125f, i13, -0.7109375f * i11))));
    v[114] = fmaf(0.001953125f, i20, fmaf(0.04296875f, i18, fmaf(-0.162109375f, i16, fmaf(0.015625f, i14, fmaf(0.66015625f, i12, -1.1171875f * i10)))));
    v[115] = fmaf(0.01953125f, i19, fmaf(0.13671875f, i17, fmaf(-0.484375f, i15, fmaf(-0.078125f, i13, 1.5234375f * i11))));
    v[116] = fmaf(0.001953125f, i20, fmaf(0.12109375f, i18, fmaf(0.462890625f, i16, fmaf(-1.296875f, i14, fmaf(-0.96484375f, i12, 3.3515625f * i10)))));
    v[117] = fmaf(0.02734375f, i19, fmaf(0.62890625f, i17, fmaf(1.859375f, i15, fmaf(-2.921875f, i13, -5.1796875f * i11))));
    v[118] = fmaf(0.001953125f, i20, fmaf(0.23046875f, i18, fmaf(3.087890625f, i16, fmaf(8.765625f, i14, fmaf(-2.58984375f, i12, -18.9921875f * i10)))));
    v[119] = fmaf(0.03515625f, i19, fmaf(1.55859375f, i17, fmaf(15.140625f, i15, fmaf(45.421875f, i13, 32.8046875f * i11))));
    v[120] = fmaf(0.001953125f, i20, fmaf(0.37109375f, i18, fmaf(9.462890625f, i16, fmaf(75.703125f, i14, fmaf(246.03515625f, i12, 360.8515625f * i10)))));
  }
};
}  // namespace jb
