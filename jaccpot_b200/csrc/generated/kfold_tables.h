// Generated by jaccpot_b200/_tables.py -- do not edit.
// In-place v <- K v with K = B^T Z0 B (the constant middle of the real
// rotate+scale M2L), block by block; indices K maps to zero are cleared.
#pragma once
namespace jb {
template <int P> struct KFold;
template <> struct KFold<1> {
  static constexpr int kNnz = 3;
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[0]; const float i3 = v[3];
      v[0] = fmaf(2.0f, i3, 1.0f * i0);
      v[3] = 2.0f * i0;
    }
    v[1] = 0.f; v[2] = 0.f;
  }
};
template <> struct KFold<2> {
  static constexpr int kNnz = 10;
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[0]; const float i3 = v[3]; const float i6 = v[6]; const float i8 = v[8];
      v[0] = fmaf(6.0f, i8, fmaf(-1.0f, i6, fmaf(2.0f, i3, 1.0f * i0)));
      v[3] = fmaf(8.0f, i3, 2.0f * i0);
      v[6] = -1.0f * i0;
      v[8] = 6.0f * i0;
    }
    {
      const float i1 = v[1];
      v[1] = -4.0f * i1;
    }
    {
      const float i2 = v[2];
      v[2] = -1.0f * i2;
    }
    v[4] = 0.f; v[5] = 0.f; v[7] = 0.f;
  }
};
template <> struct KFold<3> {
  static constexpr int kNnz = 22;
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[0]; const float i3 = v[3]; const float i6 = v[6]; const float i8 = v[8]; const float i13 = v[13]; const float i15 = v[15];
      v[0] = fmaf(30.0f, i15, fmaf(-6.0f, i13, fmaf(6.0f, i8, fmaf(-1.0f, i6, fmaf(2.0f, i3, 1.0f * i0)))));
      v[3] = fmaf(36.0f, i8, fmaf(-6.0f, i6, fmaf(8.0f, i3, 2.0f * i0)));
      v[6] = fmaf(-6.0f, i3, -1.0f * i0);
      v[8] = fmaf(36.0f, i3, 6.0f * i0);
      v[13] = -6.0f * i0;
      v[15] = 30.0f * i0;
    }
    {
      const float i1 = v[1]; const float i4 = v[4];
      v[1] = fmaf(-24.0f, i4, -4.0f * i1);
      v[4] = -24.0f * i1;
    }
    {
      const float i2 = v[2]; const float i7 = v[7];
      v[2] = fmaf(-6.0f, i7, -1.0f * i2);
      v[7] = -6.0f * i2;
    }
    v[5] = 0.f; v[9] = 0.f; v[10] = 0.f; v[11] = 0.f; v[12] = 0.f; v[14] = 0.f;
  }
};
template <> struct KFold<4> {
  static constexpr int kNnz = 47;
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[0]; const float i3 = v[3]; const float i6 = v[6]; const float i8 = v[8]; const float i13 = v[13]; const float i15 = v[15]; const float i20 = v[20]; const float i22 = v[22]; const float i24 = v[24];
      v[0] = fmaf(210.0f, i24, fmaf(-30.0f, i22, fmaf(9.0f, i20, fmaf(30.0f, i15, fmaf(-6.0f, i13, fmaf(6.0f, i8, fmaf(-1.0f, i6, fmaf(2.0f, i3, 1.0f * i0))))))));
      v[3] = fmaf(240.0f, i15, fmaf(-48.0f, i13, fmaf(36.0f, i8, fmaf(-6.0f, i6, fmaf(8.0f, i3, 2.0f * i0)))));
      v[6] = fmaf(-30.0f, i8, fmaf(9.0f, i6, fmaf(-6.0f, i3, -1.0f * i0)));
      v[8] = fmaf(228.0f, i8, fmaf(-30.0f, i6, fmaf(36.0f, i3, 6.0f * i0)));
      v[13] = fmaf(-48.0f, i3, -6.0f * i0);
      v[15] = fmaf(240.0f, i3, 30.0f * i0);
      v[20] = 9.0f * i0;
      v[22] = -30.0f * i0;
      v[24] = 210.0f * i0;
    }
    {
      const float i1 = v[1]; const float i4 = v[4]; const float i9 = v[9]; const float i11 = v[11];
      v[1] = fmaf(12.0f, i11, fmaf(-180.0f, i9, fmaf(-24.0f, i4, -4.0f * i1)));
      v[4] = fmaf(-192.0f, i4, -24.0f * i1);
      v[9] = -180.0f * i1;
      v[11] = 12.0f * i1;
    }
    {
      const float i2 = v[2]; const float i7 = v[7]; const float i12 = v[12]; const float i14 = v[14];
      v[2] = fmaf(-30.0f, i14, fmaf(9.0f, i12, fmaf(-6.0f, i7, -1.0f * i2)));
      v[7] = fmaf(-48.0f, i7, -6.0f * i2);
      v[12] = 9.0f * i2;
      v[14] = -30.0f * i2;
    }
    {
      const float i5 = v[5];
      v[5] = 12.0f * i5;
    }
    v[10] = 0.f; v[16] = 0.f; v[17] = 0.f; v[18] = 0.f; v[19] = 0.f; v[21] = 0.f; v[23] = 0.f;
  }
};
template <> struct KFold<5> {
  static constexpr int kNnz = 85;
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[0]; const float i3 = v[3]; const float i6 = v[6]; const float i8 = v[8]; const float i13 = v[13]; const float i15 = v[15]; const float i20 = v[20]; const float i22 = v[22]; const float i24 = v[24]; const float i31 = v[31]; const float i33 = v[33]; const float i35 = v[35];
      v[0] = fmaf(1890.0f, i35, fmaf(-210.0f, i33, fmaf(90.0f, i31, fmaf(210.0f, i24, fmaf(-30.0f, i22, fmaf(9.0f, i20, fmaf(30.0f, i15, fmaf(-6.0f, i13, fmaf(6.0f, i8, fmaf(-1.0f, i6, fmaf(2.0f, i3, 1.0f * i0)))))))))));
      v[3] = fmaf(2100.0f, i24, fmaf(-300.0f, i22, fmaf(90.0f, i20, fmaf(240.0f, i15, fmaf(-48.0f, i13, fmaf(36.0f, i8, fmaf(-6.0f, i6, fmaf(8.0f, i3, 2.0f * i0))))))));
      v[6] = fmaf(-210.0f, i15, fmaf(90.0f, i13, fmaf(-30.0f, i8, fmaf(9.0f, i6, fmaf(-6.0f, i3, -1.0f * i0)))));
      v[8] = fmaf(1980.0f, i15, fmaf(-300.0f, i13, fmaf(228.0f, i8, fmaf(-30.0f, i6, fmaf(36.0f, i3, 6.0f * i0)))));
      v[13] = fmaf(-300.0f, i8, fmaf(90.0f, i6, fmaf(-48.0f, i3, -6.0f * i0)));
      v[15] = fmaf(1980.0f, i8, fmaf(-210.0f, i6, fmaf(240.0f, i3, 30.0f * i0)));
      v[20] = fmaf(90.0f, i3, 9.0f * i0);
      v[22] = fmaf(-300.0f, i3, -30.0f * i0);
      v[24] = fmaf(2100.0f, i3, 210.0f * i0);
      v[31] = 90.0f * i0;
      v[33] = -210.0f * i0;
      v[35] = 1890.0f * i0;
    }
    {
      const float i1 = v[1]; const float i4 = v[4]; const float i9 = v[9]; const float i11 = v[11]; const float i16 = v[16]; const float i18 = v[18];
      v[1] = fmaf(120.0f, i18, fmaf(-1680.0f, i16, fmaf(12.0f, i11, fmaf(-180.0f, i9, fmaf(-24.0f, i4, -4.0f * i1)))));
      v[4] = fmaf(120.0f, i11, fmaf(-1800.0f, i9, fmaf(-192.0f, i4, -24.0f * i1)));
      v[9] = fmaf(-1800.0f, i4, -180.0f * i1);
      v[11] = fmaf(120.0f, i4, 12.0f * i1);
      v[16] = -1680.0f * i1;
      v[18] = 120.0f * i1;
    }
    {
      const float i2 = v[2]; const float i7 = v[7]; const float i12 = v[12]; const float i14 = v[14]; const float i21 = v[21]; const float i23 = v[23];
      v[2] = fmaf(-210.0f, i23, fmaf(90.0f, i21, fmaf(-30.0f, i14, fmaf(9.0f, i12, fmaf(-6.0f, i7, -1.0f * i2)))));
      v[7] = fmaf(-300.0f, i14, fmaf(90.0f, i12, fmaf(-48.0f, i7, -6.0f * i2)));
      v[12] = fmaf(90.0f, i7, 9.0f * i2);
      v[14] = fmaf(-300.0f, i7, -30.0f * i2);
      v[21] = 90.0f * i2;
      v[23] = -210.0f * i2;
    }
    {
      const float i5 = v[5]; const float i10 = v[10];
      v[5] = fmaf(120.0f, i10, 12.0f * i5);
      v[10] = 120.0f * i5;
    }
    v[17] = 0.f; v[19] = 0.f; v[25] = 0.f; v[26] = 0.f; v[27] = 0.f; v[28] = 0.f; v[29] = 0.f; v[30] = 0.f; v[32] = 0.f; v[34] = 0.f;
  }
};
template <> struct KFold<6> {
  static constexpr int kNnz = 148;
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[0]; const float i3 = v[3]; const float i6 = v[6]; const float i8 = v[8]; const float i13 = v[13]; const float i15 = v[15]; const float i20 = v[20]; const float i22 = v[22]; const float i24 = v[24]; const float i31 = v[31]; const float i33 = v[33]; const float i35 = v[35]; const float i42 = v[42]; const float i44 = v[44]; const float i46 = v[46]; const float i48 = v[48];
      v[0] = fmaf(20790.0f, i48, fmaf(-1890.0f, i46, fmaf(630.0f, i44, fmaf(-225.0f, i42, fmaf(1890.0f, i35, fmaf(-210.0f, i33, fmaf(90.0f, i31, fmaf(210.0f, i24, fmaf(-30.0f, i22, fmaf(9.0f, i20, fmaf(30.0f, i15, fmaf(-6.0f, i13, fmaf(6.0f, i8, fmaf(-1.0f, i6, fmaf(2.0f, i3, 1.0f * i0)))))))))))))));
      v[3] = fmaf(22680.0f, i35, fmaf(-2520.0f, i33, fmaf(1080.0f, i31, fmaf(2100.0f, i24, fmaf(-300.0f, i22, fmaf(90.0f, i20, fmaf(240.0f, i15, fmaf(-48.0f, i13, fmaf(36.0f, i8, fmaf(-6.0f, i6, fmaf(8.0f, i3, 2.0f * i0)))))))))));
      v[6] = fmaf(-1890.0f, i24, fmaf(630.0f, i22, fmaf(-225.0f, i20, fmaf(-210.0f, i15, fmaf(90.0f, i13, fmaf(-30.0f, i8, fmaf(9.0f, i6, fmaf(-6.0f, i3, -1.0f * i0))))))));
      v[8] = fmaf(21420.0f, i24, fmaf(-2340.0f, i22, fmaf(630.0f, i20, fmaf(1980.0f, i15, fmaf(-300.0f, i13, fmaf(228.0f, i8, fmaf(-30.0f, i6, fmaf(36.0f, i3, 6.0f * i0))))))));
      v[13] = fmaf(-2520.0f, i15, fmaf(1080.0f, i13, fmaf(-300.0f, i8, fmaf(90.0f, i6, fmaf(-48.0f, i3, -6.0f * i0)))));
      v[15] = fmaf(21240.0f, i15, fmaf(-2520.0f, i13, fmaf(1980.0f, i8, fmaf(-210.0f, i6, fmaf(240.0f, i3, 30.0f * i0)))));
      v[20] = fmaf(630.0f, i8, fmaf(-225.0f, i6, fmaf(90.0f, i3, 9.0f * i0)));
      v[22] = fmaf(-2340.0f, i8, fmaf(630.0f, i6, fmaf(-300.0f, i3, -30.0f * i0)));
      v[24] = fmaf(21420.0f, i8, fmaf(-1890.0f, i6, fmaf(2100.0f, i3, 210.0f * i0)));
      v[31] = fmaf(1080.0f, i3, 90.0f * i0);
      v[33] = fmaf(-2520.0f, i3, -210.0f * i0);
      v[35] = fmaf(22680.0f, i3, 1890.0f * i0);
      v[42] = -225.0f * i0;
      v[44] = 630.0f * i0;
      v[46] = -1890.0f * i0;
      v[48] = 20790.0f * i0;
    }
    {
      const float i1 = v[1]; const float i4 = v[4]; const float i9 = v[9]; const float i11 = v[11]; const float i16 = v[16]; const float i18 = v[18]; const float i25 = v[25]; const float i27 = v[27]; const float i29 = v[29];
      v[1] = fmaf(-180.0f, i29, fmaf(1260.0f, i27, fmaf(-18900.0f, i25, fmaf(120.0f, i18, fmaf(-1680.0f, i16, fmaf(12.0f, i11, fmaf(-180.0f, i9, fmaf(-24.0f, i4, -4.0f * i1))))))));
      v[4] = fmaf(1440.0f, i18, fmaf(-20160.0f, i16, fmaf(120.0f, i11, fmaf(-1800.0f, i9, fmaf(-192.0f, i4, -24.0f * i1)))));
      v[9] = fmaf(1260.0f, i11, fmaf(-20340.0f, i9, fmaf(-1800.0f, i4, -180.0f * i1)));
      v[11] = fmaf(-180.0f, i11, fmaf(1260.0f, i9, fmaf(120.0f, i4, 12.0f * i1)));
      v[16] = fmaf(-20160.0f, i4, -1680.0f * i1);
      v[18] = fmaf(1440.0f, i4, 120.0f * i1);
      v[25] = -18900.0f * i1;
      v[27] = 1260.0f * i1;
      v[29] = -180.0f * i1;
    }
    {
      const float i2 = v[2]; const float i7 = v[7]; const float i12 = v[12]; const float i14 = v[14]; const float i21 = v[21]; const float i23 = v[23]; const float i30 = v[30]; const float i32 = v[32]; const float i34 = v[34];
      v[2] = fmaf(-1890.0f, i34, fmaf(630.0f, i32, fmaf(-225.0f, i30, fmaf(-210.0f, i23, fmaf(90.0f, i21, fmaf(-30.0f, i14, fmaf(9.0f, i12, fmaf(-6.0f, i7, -1.0f * i2))))))));
      v[7] = fmaf(-2520.0f, i23, fmaf(1080.0f, i21, fmaf(-300.0f, i14, fmaf(90.0f, i12, fmaf(-48.0f, i7, -6.0f * i2)))));
      v[12] = fmaf(630.0f, i14, fmaf(-225.0f, i12, fmaf(90.0f, i7, 9.0f * i2)));
      v[14] = fmaf(-2340.0f, i14, fmaf(630.0f, i12, fmaf(-300.0f, i7, -30.0f * i2)));
      v[21] = fmaf(1080.0f, i7, 90.0f * i2);
      v[23] = fmaf(-2520.0f, i7, -210.0f * i2);
      v[30] = -225.0f * i2;
      v[32] = 630.0f * i2;
      v[34] = -1890.0f * i2;
    }
    {
      const float i5 = v[5]; const float i10 = v[10]; const float i17 = v[17]; const float i19 = v[19];
      v[5] = fmaf(-180.0f, i19, fmaf(1260.0f, i17, fmaf(120.0f, i10, 12.0f * i5)));
      v[10] = fmaf(1440.0f, i10, 120.0f * i5);
      v[17] = 1260.0f * i5;
      v[19] = -180.0f * i5;
    }
    v[26] = 0.f; v[28] = 0.f; v[36] = 0.f; v[37] = 0.f; v[38] = 0.f; v[39] = 0.f; v[40] = 0.f; v[41] = 0.f; v[43] = 0.f; v[45] = 0.f; v[47] = 0.f;
  }
};
template <> struct KFold<7> {
  static constexpr int kNnz = 236;
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[0]; const float i3 = v[3]; const float i6 = v[6]; const float i8 = v[8]; const float i13 = v[13]; const float i15 = v[15]; const float i20 = v[20]; const float i22 = v[22]; const float i24 = v[24]; const float i31 = v[31]; const float i33 = v[33]; const float i35 = v[35]; const float i42 = v[42]; const float i44 = v[44]; const float i46 = v[46]; const float i48 = v[48]; const float i57 = v[57]; const float i59 = v[59]; const float i61 = v[61]; const float i63 = v[63];
      v[0] = fmaf(270270.0f, i63, fmaf(-20790.0f, i61, fmaf(5670.0f, i59, fmaf(-3150.0f, i57, fmaf(20790.0f, i48, fmaf(-1890.0f, i46, fmaf(630.0f, i44, fmaf(-225.0f, i42, fmaf(1890.0f, i35, fmaf(-210.0f, i33, fmaf(90.0f, i31, fmaf(210.0f, i24, fmaf(-30.0f, i22, fmaf(9.0f, i20, fmaf(30.0f, i15, fmaf(-6.0f, i13, fmaf(6.0f, i8, fmaf(-1.0f, i6, fmaf(2.0f, i3, 1.0f * i0)))))))))))))))))));
      v[3] = fmaf(291060.0f, i48, fmaf(-26460.0f, i46, fmaf(8820.0f, i44, fmaf(-3150.0f, i42, fmaf(22680.0f, i35, fmaf(-2520.0f, i33, fmaf(1080.0f, i31, fmaf(2100.0f, i24, fmaf(-300.0f, i22, fmaf(90.0f, i20, fmaf(240.0f, i15, fmaf(-48.0f, i13, fmaf(36.0f, i8, fmaf(-6.0f, i6, fmaf(8.0f, i3, 2.0f * i0)))))))))))))));
      v[6] = fmaf(-20790.0f, i35, fmaf(5670.0f, i33, fmaf(-3150.0f, i31, fmaf(-1890.0f, i24, fmaf(630.0f, i22, fmaf(-225.0f, i20, fmaf(-210.0f, i15, fmaf(90.0f, i13, fmaf(-30.0f, i8, fmaf(9.0f, i6, fmaf(-6.0f, i3, -1.0f * i0)))))))))));
      v[8] = fmaf(275940.0f, i35, fmaf(-23940.0f, i33, fmaf(8820.0f, i31, fmaf(21420.0f, i24, fmaf(-2340.0f, i22, fmaf(630.0f, i20, fmaf(1980.0f, i15, fmaf(-300.0f, i13, fmaf(228.0f, i8, fmaf(-30.0f, i6, fmaf(36.0f, i3, 6.0f * i0)))))))))));
      v[13] = fmaf(-26460.0f, i24, fmaf(8820.0f, i22, fmaf(-3150.0f, i20, fmaf(-2520.0f, i15, fmaf(1080.0f, i13, fmaf(-300.0f, i8, fmaf(90.0f, i6, fmaf(-48.0f, i3, -6.0f * i0))))))));
      v[15] = fmaf(273420.0f, i24, fmaf(-23940.0f, i22, fmaf(5670.0f, i20, fmaf(21240.0f, i15, fmaf(-2520.0f, i13, fmaf(1980.0f, i8, fmaf(-210.0f, i6, fmaf(240.0f, i3, 30.0f * i0))))))));
      v[20] = fmaf(5670.0f, i15, fmaf(-3150.0f, i13, fmaf(630.0f, i8, fmaf(-225.0f, i6, fmaf(90.0f, i3, 9.0f * i0)))));
      v[22] = fmaf(-23940.0f, i15, fmaf(8820.0f, i13, fmaf(-2340.0f, i8, fmaf(630.0f, i6, fmaf(-300.0f, i3, -30.0f * i0)))));
      v[24] = fmaf(273420.0f, i15, fmaf(-26460.0f, i13, fmaf(21420.0f, i8, fmaf(-1890.0f, i6, fmaf(2100.0f, i3, 210.0f * i0)))));
      v[31] = fmaf(8820.0f, i8, fmaf(-3150.0f, i6, fmaf(1080.0f, i3, 90.0f * i0)));
      v[33] = fmaf(-23940.0f, i8, fmaf(5670.0f, i6, fmaf(-2520.0f, i3, -210.0f * i0)));
      v[35] = fmaf(275940.0f, i8, fmaf(-20790.0f, i6, fmaf(22680.0f, i3, 1890.0f * i0)));
      v[42] = fmaf(-3150.0f, i3, -225.0f * i0);
      v[44] = fmaf(8820.0f, i3, 630.0f * i0);
      v[46] = fmaf(-26460.0f, i3, -1890.0f * i0);
      v[48] = fmaf(291060.0f, i3, 20790.0f * i0);
      v[57] = -3150.0f * i0;
      v[59] = 5670.0f * i0;
      v[61] = -20790.0f * i0;
      v[63] = 270270.0f * i0;
    }
    {
      const float i1 = v[1]; const float i4 = v[4]; const float i9 = v[9]; const float i11 = v[11]; const float i16 = v[16]; const float i18 = v[18]; const float i25 = v[25]; const float i27 = v[27]; const float i29 = v[29]; const float i36 = v[36]; const float i38 = v[38]; const float i40 = v[40];
      v[1] = fmaf(-2520.0f, i40, fmaf(15120.0f, i38, fmaf(-249480.0f, i36, fmaf(-180.0f, i29, fmaf(1260.0f, i27, fmaf(-18900.0f, i25, fmaf(120.0f, i18, fmaf(-1680.0f, i16, fmaf(12.0f, i11, fmaf(-180.0f, i9, fmaf(-24.0f, i4, -4.0f * i1)))))))))));
      v[4] = fmaf(-2520.0f, i29, fmaf(17640.0f, i27, fmaf(-264600.0f, i25, fmaf(1440.0f, i18, fmaf(-20160.0f, i16, fmaf(120.0f, i11, fmaf(-1800.0f, i9, fmaf(-192.0f, i4, -24.0f * i1))))))));
      v[9] = fmaf(17640.0f, i18, fmaf(-267120.0f, i16, fmaf(1260.0f, i11, fmaf(-20340.0f, i9, fmaf(-1800.0f, i4, -180.0f * i1)))));
      v[11] = fmaf(-2520.0f, i18, fmaf(15120.0f, i16, fmaf(-180.0f, i11, fmaf(1260.0f, i9, fmaf(120.0f, i4, 12.0f * i1)))));
      v[16] = fmaf(15120.0f, i11, fmaf(-267120.0f, i9, fmaf(-20160.0f, i4, -1680.0f * i1)));
      v[18] = fmaf(-2520.0f, i11, fmaf(17640.0f, i9, fmaf(1440.0f, i4, 120.0f * i1)));
      v[25] = fmaf(-264600.0f, i4, -18900.0f * i1);
      v[27] = fmaf(17640.0f, i4, 1260.0f * i1);
      v[29] = fmaf(-2520.0f, i4, -180.0f * i1);
      v[36] = -249480.0f * i1;
      v[38] = 15120.0f * i1;
      v[40] = -2520.0f * i1;
    }
    {
      const float i2 = v[2]; const float i7 = v[7]; const float i12 = v[12]; const float i14 = v[14]; const float i21 = v[21]; const float i23 = v[23]; const float i30 = v[30]; const float i32 = v[32]; const float i34 = v[34]; const float i43 = v[43]; const float i45 = v[45]; const float i47 = v[47];
      v[2] = fmaf(-20790.0f, i47, fmaf(5670.0f, i45, fmaf(-3150.0f, i43, fmaf(-1890.0f, i34, fmaf(630.0f, i32, fmaf(-225.0f, i30, fmaf(-210.0f, i23, fmaf(90.0f, i21, fmaf(-30.0f, i14, fmaf(9.0f, i12, fmaf(-6.0f, i7, -1.0f * i2)))))))))));
      v[7] = fmaf(-26460.0f, i34, fmaf(8820.0f, i32, fmaf(-3150.0f, i30, fmaf(-2520.0f, i23, fmaf(1080.0f, i21, fmaf(-300.0f, i14, fmaf(90.0f, i12, fmaf(-48.0f, i7, -6.0f * i2))))))));
      v[12] = fmaf(5670.0f, i23, fmaf(-3150.0f, i21, fmaf(630.0f, i14, fmaf(-225.0f, i12, fmaf(90.0f, i7, 9.0f * i2)))));
      v[14] = fmaf(-23940.0f, i23, fmaf(8820.0f, i21, fmaf(-2340.0f, i14, fmaf(630.0f, i12, fmaf(-300.0f, i7, -30.0f * i2)))));
      v[21] = fmaf(8820.0f, i14, fmaf(-3150.0f, i12, fmaf(1080.0f, i7, 90.0f * i2)));
      v[23] = fmaf(-23940.0f, i14, fmaf(5670.0f, i12, fmaf(-2520.0f, i7, -210.0f * i2)));
      v[30] = fmaf(-3150.0f, i7, -225.0f * i2);
      v[32] = fmaf(8820.0f, i7, 630.0f * i2);
      v[34] = fmaf(-26460.0f, i7, -1890.0f * i2);
      v[43] = -3150.0f * i2;
      v[45] = 5670.0f * i2;
      v[47] = -20790.0f * i2;
    }
    {
      const float i5 = v[5]; const float i10 = v[10]; const float i17 = v[17]; const float i19 = v[19]; const float i26 = v[26]; const float i28 = v[28];
      v[5] = fmaf(-2520.0f, i28, fmaf(15120.0f, i26, fmaf(-180.0f, i19, fmaf(1260.0f, i17, fmaf(120.0f, i10, 12.0f * i5)))));
      v[10] = fmaf(-2520.0f, i19, fmaf(17640.0f, i17, fmaf(1440.0f, i10, 120.0f * i5)));
      v[17] = fmaf(17640.0f, i10, 1260.0f * i5);
      v[19] = fmaf(-2520.0f, i10, -180.0f * i5);
      v[26] = 15120.0f * i5;
      v[28] = -2520.0f * i5;
    }
    v[37] = 0.f; v[39] = 0.f; v[41] = 0.f; v[49] = 0.f; v[50] = 0.f; v[51] = 0.f; v[52] = 0.f; v[53] = 0.f; v[54] = 0.f; v[55] = 0.f; v[56] = 0.f; v[58] = 0.f; v[60] = 0.f; v[62] = 0.f;
  }
};
template <> struct KFold<8> {
  static constexpr int kNnz = 365;
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[0]; const float i3 = v[3]; const float i6 = v[6]; const float i8 = v[8]; const float i13 = v[13]; const float i15 = v[15]; const float i20 = v[20]; const float i22 = v[22]; const float i24 = v[24]; const float i31 = v[31]; const float i33 = v[33]; const float i35 = v[35]; const float i42 = v[42]; const float i44 = v[44]; const float i46 = v[46]; const float i48 = v[48]; const float i57 = v[57]; const float i59 = v[59]; const float i61 = v[61]; const float i63 = v[63]; const float i72 = v[72]; const float i74 = v[74]; const float i76 = v[76]; const float i78 = v[78]; const float i80 = v[80];
      v[0] = fmaf(4054050.0f, i80, fmaf(-270270.0f, i78, fmaf(62370.0f, i76, fmaf(-28350.0f, i74, fmaf(11025.0f, i72, fmaf(270270.0f, i63, fmaf(-20790.0f, i61, fmaf(5670.0f, i59, fmaf(-3150.0f, i57, fmaf(20790.0f, i48, fmaf(-1890.0f, i46, fmaf(630.0f, i44, fmaf(-225.0f, i42, fmaf(1890.0f, i35, fmaf(-210.0f, i33, fmaf(90.0f, i31, fmaf(210.0f, i24, fmaf(-30.0f, i22, fmaf(9.0f, i20, fmaf(30.0f, i15, fmaf(-6.0f, i13, fmaf(6.0f, i8, fmaf(-1.0f, i6, fmaf(2.0f, i3, 1.0f * i0))))))))))))))))))))))));
      v[3] = fmaf(4324320.0f, i63, fmaf(-332640.0f, i61, fmaf(90720.0f, i59, fmaf(-50400.0f, i57, fmaf(291060.0f, i48, fmaf(-26460.0f, i46, fmaf(8820.0f, i44, fmaf(-3150.0f, i42, fmaf(22680.0f, i35, fmaf(-2520.0f, i33, fmaf(1080.0f, i31, fmaf(2100.0f, i24, fmaf(-300.0f, i22, fmaf(90.0f, i20, fmaf(240.0f, i15, fmaf(-48.0f, i13, fmaf(36.0f, i8, fmaf(-6.0f, i6, fmaf(8.0f, i3, 2.0f * i0)))))))))))))))))));
      v[6] = fmaf(-270270.0f, i48, fmaf(62370.0f, i46, fmaf(-28350.0f, i44, fmaf(11025.0f, i42, fmaf(-20790.0f, i35, fmaf(5670.0f, i33, fmaf(-3150.0f, i31, fmaf(-1890.0f, i24, fmaf(630.0f, i22, fmaf(-225.0f, i20, fmaf(-210.0f, i15, fmaf(90.0f, i13, fmaf(-30.0f, i8, fmaf(9.0f, i6, fmaf(-6.0f, i3, -1.0f * i0)))))))))))))));
      v[8] = fmaf(4116420.0f, i48, fmaf(-298620.0f, i46, fmaf(84420.0f, i44, fmaf(-28350.0f, i42, fmaf(275940.0f, i35, fmaf(-23940.0f, i33, fmaf(8820.0f, i31, fmaf(21420.0f, i24, fmaf(-2340.0f, i22, fmaf(630.0f, i20, fmaf(1980.0f, i15, fmaf(-300.0f, i13, fmaf(228.0f, i8, fmaf(-30.0f, i6, fmaf(36.0f, i3, 6.0f * i0)))))))))))))));
      v[13] = fmaf(-332640.0f, i35, fmaf(90720.0f, i33, fmaf(-50400.0f, i31, fmaf(-26460.0f, i24, fmaf(8820.0f, i22, fmaf(-3150.0f, i20, fmaf(-2520.0f, i15, fmaf(1080.0f, i13, fmaf(-300.0f, i8, fmaf(90.0f, i6, fmaf(-48.0f, i3, -6.0f * i0)))))))))));
      v[15] = fmaf(4082400.0f, i35, fmaf(-292320.0f, i33, fmaf(90720.0f, i31, fmaf(273420.0f, i24, fmaf(-23940.0f, i22, fmaf(5670.0f, i20, fmaf(21240.0f, i15, fmaf(-2520.0f, i13, fmaf(1980.0f, i8, fmaf(-210.0f, i6, fmaf(240.0f, i3, 30.0f * i0)))))))))));
      v[20] = fmaf(62370.0f, i24, fmaf(-28350.0f, i22, fmaf(11025.0f, i20, fmaf(5670.0f, i15, fmaf(-3150.0f, i13, fmaf(630.0f, i8, fmaf(-225.0f, i6, fmaf(90.0f, i3, 9.0f * i0))))))));
      v[22] = fmaf(-298620.0f, i24, fmaf(84420.0f, i22, fmaf(-28350.0f, i20, fmaf(-23940.0f, i15, fmaf(8820.0f, i13, fmaf(-2340.0f, i8, fmaf(630.0f, i6, fmaf(-300.0f, i3, -30.0f * i0))))))));
      v[24] = fmaf(4076100.0f, i24, fmaf(-298620.0f, i22, fmaf(62370.0f, i20, fmaf(273420.0f, i15, fmaf(-26460.0f, i13, fmaf(21420.0f, i8, fmaf(-1890.0f, i6, fmaf(2100.0f, i3, 210.0f * i0))))))));
      v[31] = fmaf(90720.0f, i15, fmaf(-50400.0f, i13, fmaf(8820.0f, i8, fmaf(-3150.0f, i6, fmaf(1080.0f, i3, 90.0f * i0)))));
      v[33] = fmaf(-292320.0f, i15, fmaf(90720.0f, i13, fmaf(-23940.0f, i8, fmaf(5670.0f, i6, fmaf(-2520.0f, i3, -210.0f * i0)))));
      v[35] = fmaf(4082400.0f, i15, fmaf(-332640.0f, i13, fmaf(275940.0f, i8, fmaf(-20790.0f, i6, fmaf(22680.0f, i3, 1890.0f * i0)))));
      v[42] = fmaf(-28350.0f, i8, fmaf(11025.0f, i6, fmaf(-3150.0f, i3, -225.0f * i0)));
      v[44] = fmaf(84420.0f, i8, fmaf(-28350.0f, i6, fmaf(8820.0f, i3, 630.0f * i0)));
      v[46] = fmaf(-298620.0f, i8, fmaf(62370.0f, i6, fmaf(-26460.0f, i3, -1890.0f * i0)));
      v[48] = fmaf(4116420.0f, i8, fmaf(-270270.0f, i6, fmaf(291060.0f, i3, 20790.0f * i0)));
      v[57] = fmaf(-50400.0f, i3, -3150.0f * i0);
      v[59] = fmaf(90720.0f, i3, 5670.0f * i0);
      v[61] = fmaf(-332640.0f, i3, -20790.0f * i0);
      v[63] = fmaf(4324320.0f, i3, 270270.0f * i0);
      v[72] = 11025.0f * i0;
      v[74] = -28350.0f * i0;
      v[76] = 62370.0f * i0;
      v[78] = -270270.0f * i0;
      v[80] = 4054050.0f * i0;
    }
    {
      const float i1 = v[1]; const float i4 = v[4]; const float i9 = v[9]; const float i11 = v[11]; const float i16 = v[16]; const float i18 = v[18]; const float i25 = v[25]; const float i27 = v[27]; const float i29 = v[29]; const float i36 = v[36]; const float i38 = v[38]; const float i40 = v[40]; const float i49 = v[49]; const float i51 = v[51]; const float i53 = v[53]; const float i55 = v[55];
      v[1] = fmaf(6300.0f, i55, fmaf(-34020.0f, i53, fmaf(207900.0f, i51, fmaf(-3783780.0f, i49, fmaf(-2520.0f, i40, fmaf(15120.0f, i38, fmaf(-249480.0f, i36, fmaf(-180.0f, i29, fmaf(1260.0f, i27, fmaf(-18900.0f, i25, fmaf(120.0f, i18, fmaf(-1680.0f, i16, fmaf(12.0f, i11, fmaf(-180.0f, i9, fmaf(-24.0f, i4, -4.0f * i1)))))))))))))));
      v[4] = fmaf(-40320.0f, i40, fmaf(241920.0f, i38, fmaf(-3991680.0f, i36, fmaf(-2520.0f, i29, fmaf(17640.0f, i27, fmaf(-264600.0f, i25, fmaf(1440.0f, i18, fmaf(-20160.0f, i16, fmaf(120.0f, i11, fmaf(-1800.0f, i9, fmaf(-192.0f, i4, -24.0f * i1)))))))))));
      v[9] = fmaf(-34020.0f, i29, fmaf(248220.0f, i27, fmaf(-4025700.0f, i25, fmaf(17640.0f, i18, fmaf(-267120.0f, i16, fmaf(1260.0f, i11, fmaf(-20340.0f, i9, fmaf(-1800.0f, i4, -180.0f * i1))))))));
      v[11] = fmaf(6300.0f, i29, fmaf(-34020.0f, i27, fmaf(207900.0f, i25, fmaf(-2520.0f, i18, fmaf(15120.0f, i16, fmaf(-180.0f, i11, fmaf(1260.0f, i9, fmaf(120.0f, i4, 12.0f * i1))))))));
      v[16] = fmaf(241920.0f, i18, fmaf(-4032000.0f, i16, fmaf(15120.0f, i11, fmaf(-267120.0f, i9, fmaf(-20160.0f, i4, -1680.0f * i1)))));
      v[18] = fmaf(-40320.0f, i18, fmaf(241920.0f, i16, fmaf(-2520.0f, i11, fmaf(17640.0f, i9, fmaf(1440.0f, i4, 120.0f * i1)))));
      v[25] = fmaf(207900.0f, i11, fmaf(-4025700.0f, i9, fmaf(-264600.0f, i4, -18900.0f * i1)));
      v[27] = fmaf(-34020.0f, i11, fmaf(248220.0f, i9, fmaf(17640.0f, i4, 1260.0f * i1)));
      v[29] = fmaf(6300.0f, i11, fmaf(-34020.0f, i9, fmaf(-2520.0f, i4, -180.0f * i1)));
      v[36] = fmaf(-3991680.0f, i4, -249480.0f * i1);
      v[38] = fmaf(241920.0f, i4, 15120.0f * i1);
      v[40] = fmaf(-40320.0f, i4, -2520.0f * i1);
      v[49] = -3783780.0f * i1;
      v[51] = 207900.0f * i1;
      v[53] = -34020.0f * i1;
      v[55] = 6300.0f * i1;
    }
    {
      const float i2 = v[2]; const float i7 = v[7]; const float i12 = v[12]; const float i14 = v[14]; const float i21 = v[21]; const float i23 = v[23]; const float i30 = v[30]; const float i32 = v[32]; const float i34 = v[34]; const float i43 = v[43]; const float i45 = v[45]; const float i47 = v[47]; const float i56 = v[56]; const float i58 = v[58]; const float i60 = v[60]; const float i62 = v[62];
      v[2] = fmaf(-270270.0f, i62, fmaf(62370.0f, i60, fmaf(-28350.0f, i58, fmaf(11025.0f, i56, fmaf(-20790.0f, i47, fmaf(5670.0f, i45, fmaf(-3150.0f, i43, fmaf(-1890.0f, i34, fmaf(630.0f, i32, fmaf(-225.0f, i30, fmaf(-210.0f, i23, fmaf(90.0f, i21, fmaf(-30.0f, i14, fmaf(9.0f, i12, fmaf(-6.0f, i7, -1.0f * i2)))))))))))))));
      v[7] = fmaf(-332640.0f, i47, fmaf(90720.0f, i45, fmaf(-50400.0f, i43, fmaf(-26460.0f, i34, fmaf(8820.0f, i32, fmaf(-3150.0f, i30, fmaf(-2520.0f, i23, fmaf(1080.0f, i21, fmaf(-300.0f, i14, fmaf(90.0f, i12, fmaf(-48.0f, i7, -6.0f * i2)))))))))));
      v[12] = fmaf(62370.0f, i34, fmaf(-28350.0f, i32, fmaf(11025.0f, i30, fmaf(5670.0f, i23, fmaf(-3150.0f, i21, fmaf(630.0f, i14, fmaf(-225.0f, i12, fmaf(90.0f, i7, 9.0f * i2))))))));
      v[14] = fmaf(-298620.0f, i34, fmaf(84420.0f, i32, fmaf(-28350.0f, i30, fmaf(-23940.0f, i23, fmaf(8820.0f, i21, fmaf(-2340.0f, i14, fmaf(630.0f, i12, fmaf(-300.0f, i7, -30.0f * i2))))))));
      v[21] = fmaf(90720.0f, i23, fmaf(-50400.0f, i21, fmaf(8820.0f, i14, fmaf(-3150.0f, i12, fmaf(1080.0f, i7, 90.0f * i2)))));
      v[23] = fmaf(-292320.0f, i23, fmaf(90720.0f, i21, fmaf(-23940.0f, i14, fmaf(5670.0f, i12, fmaf(-2520.0f, i7, -210.0f * i2)))));
      v[30] = fmaf(-28350.0f, i14, fmaf(11025.0f, i12, fmaf(-3150.0f, i7, -225.0f * i2)));
      v[32] = fmaf(84420.0f, i14, fmaf(-28350.0f, i12, fmaf(8820.0f, i7, 630.0f * i2)));
      v[34] = fmaf(-298620.0f, i14, fmaf(62370.0f, i12, fmaf(-26460.0f, i7, -1890.0f * i2)));
      v[43] = fmaf(-50400.0f, i7, -3150.0f * i2);
      v[45] = fmaf(90720.0f, i7, 5670.0f * i2);
      v[47] = fmaf(-332640.0f, i7, -20790.0f * i2);
      v[56] = 11025.0f * i2;
      v[58] = -28350.0f * i2;
      v[60] = 62370.0f * i2;
      v[62] = -270270.0f * i2;
    }
    {
      const float i5 = v[5]; const float i10 = v[10]; const float i17 = v[17]; const float i19 = v[19]; const float i26 = v[26]; const float i28 = v[28]; const float i37 = v[37]; const float i39 = v[39]; const float i41 = v[41];
      v[5] = fmaf(6300.0f, i41, fmaf(-34020.0f, i39, fmaf(207900.0f, i37, fmaf(-2520.0f, i28, fmaf(15120.0f, i26, fmaf(-180.0f, i19, fmaf(1260.0f, i17, fmaf(120.0f, i10, 12.0f * i5))))))));
      v[10] = fmaf(-40320.0f, i28, fmaf(241920.0f, i26, fmaf(-2520.0f, i19, fmaf(17640.0f, i17, fmaf(1440.0f, i10, 120.0f * i5)))));
      v[17] = fmaf(-34020.0f, i19, fmaf(248220.0f, i17, fmaf(17640.0f, i10, 1260.0f * i5)));
      v[19] = fmaf(6300.0f, i19, fmaf(-34020.0f, i17, fmaf(-2520.0f, i10, -180.0f * i5)));
      v[26] = fmaf(241920.0f, i10, 15120.0f * i5);
      v[28] = fmaf(-40320.0f, i10, -2520.0f * i5);
      v[37] = 207900.0f * i5;
      v[39] = -34020.0f * i5;
      v[41] = 6300.0f * i5;
    }
    v[50] = 0.f; v[52] = 0.f; v[54] = 0.f; v[64] = 0.f; v[65] = 0.f; v[66] = 0.f; v[67] = 0.f; v[68] = 0.f; v[69] = 0.f; v[70] = 0.f; v[71] = 0.f; v[73] = 0.f; v[75] = 0.f; v[77] = 0.f; v[79] = 0.f;
  }
};
template <> struct KFold<9> {
  static constexpr int kNnz = 535;
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[0]; const float i3 = v[3]; const float i6 = v[6]; const float i8 = v[8]; const float i13 = v[13]; const float i15 = v[15]; const float i20 = v[20]; const float i22 = v[22]; const float i24 = v[24]; const float i31 = v[31]; const float i33 = v[33]; const float i35 = v[35]; const float i42 = v[42]; const float i44 = v[44]; const float i46 = v[46]; const float i48 = v[48]; const float i57 = v[57]; const float i59 = v[59]; const float i61 = v[61]; const float i63 = v[63]; const float i72 = v[72]; const float i74 = v[74]; const float i76 = v[76]; const float i78 = v[78]; const float i80 = v[80]; const float i91 = v[91]; const float i93 = v[93]; const float i95 = v[95]; const float i97 = v[97]; const float i99 = v[99];
      v[0] = fmaf(68918848.0f, i99, fmaf(-4054050.0f, i97, fmaf(810810.0f, i95, fmaf(-311850.0f, i93, fmaf(198450.0f, i91, fmaf(4054050.0f, i80, fmaf(-270270.0f, i78, fmaf(62370.0f, i76, fmaf(-28350.0f, i74, fmaf(11025.0f, i72, fmaf(270270.0f, i63, fmaf(-20790.0f, i61, fmaf(5670.0f, i59, fmaf(-3150.0f, i57, fmaf(20790.0f, i48, fmaf(-1890.0f, i46, fmaf(630.0f, i44, fmaf(-225.0f, i42, fmaf(1890.0f, i35, fmaf(-210.0f, i33, fmaf(90.0f, i31, fmaf(210.0f, i24, fmaf(-30.0f, i22, fmaf(9.0f, i20, fmaf(30.0f, i15, fmaf(-6.0f, i13, fmaf(6.0f, i8, fmaf(-1.0f, i6, fmaf(2.0f, i3, 1.0f * i0)))))))))))))))))))))))))))));
      v[3] = fmaf(72972896.0f, i80, fmaf(-4864860.0f, i78, fmaf(1122660.0f, i76, fmaf(-510300.0f, i74, fmaf(198450.0f, i72, fmaf(4324320.0f, i63, fmaf(-332640.0f, i61, fmaf(90720.0f, i59, fmaf(-50400.0f, i57, fmaf(291060.0f, i48, fmaf(-26460.0f, i46, fmaf(8820.0f, i44, fmaf(-3150.0f, i42, fmaf(22680.0f, i35, fmaf(-2520.0f, i33, fmaf(1080.0f, i31, fmaf(2100.0f, i24, fmaf(-300.0f, i22, fmaf(90.0f, i20, fmaf(240.0f, i15, fmaf(-48.0f, i13, fmaf(36.0f, i8, fmaf(-6.0f, i6, fmaf(8.0f, i3, 2.0f * i0))))))))))))))))))))))));
      v[6] = fmaf(-4054050.0f, i63, fmaf(810810.0f, i61, fmaf(-311850.0f, i59, fmaf(198450.0f, i57, fmaf(-270270.0f, i48, fmaf(62370.0f, i46, fmaf(-28350.0f, i44, fmaf(11025.0f, i42, fmaf(-20790.0f, i35, fmaf(5670.0f, i33, fmaf(-3150.0f, i31, fmaf(-1890.0f, i24, fmaf(630.0f, i22, fmaf(-225.0f, i20, fmaf(-210.0f, i15, fmaf(90.0f, i13, fmaf(-30.0f, i8, fmaf(9.0f, i6, fmaf(-6.0f, i3, -1.0f * i0)))))))))))))))))));
      v[8] = fmaf(69729664.0f, i63, fmaf(-4365900.0f, i61, fmaf(1009260.0f, i59, fmaf(-510300.0f, i57, fmaf(4116420.0f, i48, fmaf(-298620.0f, i46, fmaf(84420.0f, i44, fmaf(-28350.0f, i42, fmaf(275940.0f, i35, fmaf(-23940.0f, i33, fmaf(8820.0f, i31, fmaf(21420.0f, i24, fmaf(-2340.0f, i22, fmaf(630.0f, i20, fmaf(1980.0f, i15, fmaf(-300.0f, i13, fmaf(228.0f, i8, fmaf(-30.0f, i6, fmaf(36.0f, i3, 6.0f * i0)))))))))))))))))));
      v[13] = fmaf(-4864860.0f, i48, fmaf(1122660.0f, i46, fmaf(-510300.0f, i44, fmaf(198450.0f, i42, fmaf(-332640.0f, i35, fmaf(90720.0f, i33, fmaf(-50400.0f, i31, fmaf(-26460.0f, i24, fmaf(8820.0f, i22, fmaf(-3150.0f, i20, fmaf(-2520.0f, i15, fmaf(1080.0f, i13, fmaf(-300.0f, i8, fmaf(90.0f, i6, fmaf(-48.0f, i3, -6.0f * i0)))))))))))))));
      v[15] = fmaf(69230704.0f, i48, fmaf(-4252500.0f, i46, fmaf(1009260.0f, i44, fmaf(-311850.0f, i42, fmaf(4082400.0f, i35, fmaf(-292320.0f, i33, fmaf(90720.0f, i31, fmaf(273420.0f, i24, fmaf(-23940.0f, i22, fmaf(5670.0f, i20, fmaf(21240.0f, i15, fmaf(-2520.0f, i13, fmaf(1980.0f, i8, fmaf(-210.0f, i6, fmaf(240.0f, i3, 30.0f * i0)))))))))))))));
      v[20] = fmaf(810810.0f, i35, fmaf(-311850.0f, i33, fmaf(198450.0f, i31, fmaf(62370.0f, i24, fmaf(-28350.0f, i22, fmaf(11025.0f, i20, fmaf(5670.0f, i15, fmaf(-3150.0f, i13, fmaf(630.0f, i8, fmaf(-225.0f, i6, fmaf(90.0f, i3, 9.0f * i0)))))))))));
      v[22] = fmaf(-4365900.0f, i35, fmaf(1009260.0f, i33, fmaf(-510300.0f, i31, fmaf(-298620.0f, i24, fmaf(84420.0f, i22, fmaf(-28350.0f, i20, fmaf(-23940.0f, i15, fmaf(8820.0f, i13, fmaf(-2340.0f, i8, fmaf(630.0f, i6, fmaf(-300.0f, i3, -30.0f * i0)))))))))));
      v[24] = fmaf(69117296.0f, i35, fmaf(-4252500.0f, i33, fmaf(1122660.0f, i31, fmaf(4076100.0f, i24, fmaf(-298620.0f, i22, fmaf(62370.0f, i20, fmaf(273420.0f, i15, fmaf(-26460.0f, i13, fmaf(21420.0f, i8, fmaf(-1890.0f, i6, fmaf(2100.0f, i3, 210.0f * i0)))))))))));
      v[31] = fmaf(1122660.0f, i24, fmaf(-510300.0f, i22, fmaf(198450.0f, i20, fmaf(90720.0f, i15, fmaf(-50400.0f, i13, fmaf(8820.0f, i8, fmaf(-3150.0f, i6, fmaf(1080.0f, i3, 90.0f * i0))))))));
      v[33] = fmaf(-4252500.0f, i24, fmaf(1009260.0f, i22, fmaf(-311850.0f, i20, fmaf(-292320.0f, i15, fmaf(90720.0f, i13, fmaf(-23940.0f, i8, fmaf(5670.0f, i6, fmaf(-2520.0f, i3, -210.0f * i0))))))));
      v[35] = fmaf(69117296.0f, i24, fmaf(-4365900.0f, i22, fmaf(810810.0f, i20, fmaf(4082400.0f, i15, fmaf(-332640.0f, i13, fmaf(275940.0f, i8, fmaf(-20790.0f, i6, fmaf(22680.0f, i3, 1890.0f * i0))))))));
      v[42] = fmaf(-311850.0f, i15, fmaf(198450.0f, i13, fmaf(-28350.0f, i8, fmaf(11025.0f, i6, fmaf(-3150.0f, i3, -225.0f * i0)))));
      v[44] = fmaf(1009260.0f, i15, fmaf(-510300.0f, i13, fmaf(84420.0f, i8, fmaf(-28350.0f, i6, fmaf(8820.0f, i3, 630.0f * i0)))));
      v[46] = fmaf(-4252500.0f, i15, fmaf(1122660.0f, i13, fmaf(-298620.0f, i8, fmaf(62370.0f, i6, fmaf(-26460.0f, i3, -1890.0f * i0)))));
      v[48] = fmaf(69230704.0f, i15, fmaf(-4864860.0f, i13, fmaf(4116420.0f, i8, fmaf(-270270.0f, i6, fmaf(291060.0f, i3, 20790.0f * i0)))));
      v[57] = fmaf(-510300.0f, i8, fmaf(198450.0f, i6, fmaf(-50400.0f, i3, -3150.0f * i0)));
      v[59] = fmaf(1009260.0f, i8, fmaf(-311850.0f, i6, fmaf(90720.0f, i3, 5670.0f * i0)));
      v[61] = fmaf(-4365900.0f, i8, fmaf(810810.0f, i6, fmaf(-332640.0f, i3, -20790.0f * i0)));
      v[63] = fmaf(69729664.0f, i8, fmaf(-4054050.0f, i6, fmaf(4324320.0f, i3, 270270.0f * i0)));
      v[72] = fmaf(198450.0f, i3, 11025.0f * i0);
      v[74] = fmaf(-510300.0f, i3, -28350.0f * i0);
      v[76] = fmaf(1122660.0f, i3, 62370.0f * i0);
      v[78] = fmaf(-4864860.0f, i3, -270270.0f * i0);
      v[80] = fmaf(72972896.0f, i3, 4054050.0f * i0);
      v[91] = 198450.0f * i0;
      v[93] = -311850.0f * i0;
      v[95] = 810810.0f * i0;
      v[97] = -4054050.0f * i0;
      v[99] = 68918848.0f * i0;
    }
    {
      const float i1 = v[1]; const float i4 = v[4]; const float i9 = v[9]; const float i11 = v[11]; const float i16 = v[16]; const float i18 = v[18]; const float i25 = v[25]; const float i27 = v[27]; const float i29 = v[29]; const float i36 = v[36]; const float i38 = v[38]; const float i40 = v[40]; const float i49 = v[49]; const float i51 = v[51]; const float i53 = v[53]; const float i55 = v[55]; const float i64 = v[64]; const float i66 = v[66]; const float i68 = v[68]; const float i70 = v[70];
      v[1] = fmaf(113400.0f, i70, fmaf(-498960.0f, i68, fmaf(3243240.0f, i66, fmaf(-64864800.0f, i64, fmaf(6300.0f, i55, fmaf(-34020.0f, i53, fmaf(207900.0f, i51, fmaf(-3783780.0f, i49, fmaf(-2520.0f, i40, fmaf(15120.0f, i38, fmaf(-249480.0f, i36, fmaf(-180.0f, i29, fmaf(1260.0f, i27, fmaf(-18900.0f, i25, fmaf(120.0f, i18, fmaf(-1680.0f, i16, fmaf(12.0f, i11, fmaf(-180.0f, i9, fmaf(-24.0f, i4, -4.0f * i1)))))))))))))))))));
      v[4] = fmaf(113400.0f, i55, fmaf(-612360.0f, i53, fmaf(3742200.0f, i51, fmaf(-68108040.0f, i49, fmaf(-40320.0f, i40, fmaf(241920.0f, i38, fmaf(-3991680.0f, i36, fmaf(-2520.0f, i29, fmaf(17640.0f, i27, fmaf(-264600.0f, i25, fmaf(1440.0f, i18, fmaf(-20160.0f, i16, fmaf(120.0f, i11, fmaf(-1800.0f, i9, fmaf(-192.0f, i4, -24.0f * i1)))))))))))))));
      v[9] = fmaf(-612360.0f, i40, fmaf(3855600.0f, i38, fmaf(-68607000.0f, i36, fmaf(-34020.0f, i29, fmaf(248220.0f, i27, fmaf(-4025700.0f, i25, fmaf(17640.0f, i18, fmaf(-267120.0f, i16, fmaf(1260.0f, i11, fmaf(-20340.0f, i9, fmaf(-1800.0f, i4, -180.0f * i1)))))))))));
      v[11] = fmaf(113400.0f, i40, fmaf(-498960.0f, i38, fmaf(3243240.0f, i36, fmaf(6300.0f, i29, fmaf(-34020.0f, i27, fmaf(207900.0f, i25, fmaf(-2520.0f, i18, fmaf(15120.0f, i16, fmaf(-180.0f, i11, fmaf(1260.0f, i9, fmaf(120.0f, i4, 12.0f * i1)))))))))));
      v[16] = fmaf(-498960.0f, i29, fmaf(3855600.0f, i27, fmaf(-68720400.0f, i25, fmaf(241920.0f, i18, fmaf(-4032000.0f, i16, fmaf(15120.0f, i11, fmaf(-267120.0f, i9, fmaf(-20160.0f, i4, -1680.0f * i1))))))));
      v[18] = fmaf(113400.0f, i29, fmaf(-612360.0f, i27, fmaf(3742200.0f, i25, fmaf(-40320.0f, i18, fmaf(241920.0f, i16, fmaf(-2520.0f, i11, fmaf(17640.0f, i9, fmaf(1440.0f, i4, 120.0f * i1))))))));
      v[25] = fmaf(3742200.0f, i18, fmaf(-68720400.0f, i16, fmaf(207900.0f, i11, fmaf(-4025700.0f, i9, fmaf(-264600.0f, i4, -18900.0f * i1)))));
      v[27] = fmaf(-612360.0f, i18, fmaf(3855600.0f, i16, fmaf(-34020.0f, i11, fmaf(248220.0f, i9, fmaf(17640.0f, i4, 1260.0f * i1)))));
      v[29] = fmaf(113400.0f, i18, fmaf(-498960.0f, i16, fmaf(6300.0f, i11, fmaf(-34020.0f, i9, fmaf(-2520.0f, i4, -180.0f * i1)))));
      v[36] = fmaf(3243240.0f, i11, fmaf(-68607000.0f, i9, fmaf(-3991680.0f, i4, -249480.0f * i1)));
      v[38] = fmaf(-498960.0f, i11, fmaf(3855600.0f, i9, fmaf(241920.0f, i4, 15120.0f * i1)));
      v[40] = fmaf(113400.0f, i11, fmaf(-612360.0f, i9, fmaf(-40320.0f, i4, -2520.0f * i1)));
      v[49] = fmaf(-68108040.0f, i4, -3783780.0f * i1);
      v[51] = fmaf(3742200.0f, i4, 207900.0f * i1);
      v[53] = fmaf(-612360.0f, i4, -34020.0f * i1);
      v[55] = fmaf(113400.0f, i4, 6300.0f * i1);
      v[64] = -64864800.0f * i1;
      v[66] = 3243240.0f * i1;
      v[68] = -498960.0f * i1;
      v[70] = 113400.0f * i1;
    }
    {
      const float i2 = v[2]; const float i7 = v[7]; const float i12 = v[12]; const float i14 = v[14]; const float i21 = v[21]; const float i23 = v[23]; const float i30 = v[30]; const float i32 = v[32]; const float i34 = v[34]; const float i43 = v[43]; const float i45 = v[45]; const float i47 = v[47]; const float i56 = v[56]; const float i58 = v[58]; const float i60 = v[60]; const float i62 = v[62]; const float i73 = v[73]; const float i75 = v[75]; const float i77 = v[77]; const float i79 = v[79];
      v[2] = fmaf(-4054050.0f, i79, fmaf(810810.0f, i77, fmaf(-311850.0f, i75, fmaf(198450.0f, i73, fmaf(-270270.0f, i62, fmaf(62370.0f, i60, fmaf(-28350.0f, i58, fmaf(11025.0f, i56, fmaf(-20790.0f, i47, fmaf(5670.0f, i45, fmaf(-3150.0f, i43, fmaf(-1890.0f, i34, fmaf(630.0f, i32, fmaf(-225.0f, i30, fmaf(-210.0f, i23, fmaf(90.0f, i21, fmaf(-30.0f, i14, fmaf(9.0f, i12, fmaf(-6.0f, i7, -1.0f * i2)))))))))))))))))));
      v[7] = fmaf(-4864860.0f, i62, fmaf(1122660.0f, i60, fmaf(-510300.0f, i58, fmaf(198450.0f, i56, fmaf(-332640.0f, i47, fmaf(90720.0f, i45, fmaf(-50400.0f, i43, fmaf(-26460.0f, i34, fmaf(8820.0f, i32, fmaf(-3150.0f, i30, fmaf(-2520.0f, i23, fmaf(1080.0f, i21, fmaf(-300.0f, i14, fmaf(90.0f, i12, fmaf(-48.0f, i7, -6.0f * i2)))))))))))))));
      v[12] = fmaf(810810.0f, i47, fmaf(-311850.0f, i45, fmaf(198450.0f, i43, fmaf(62370.0f, i34, fmaf(-28350.0f, i32, fmaf(11025.0f, i30, fmaf(5670.0f, i23, fmaf(-3150.0f, i21, fmaf(630.0f, i14, fmaf(-225.0f, i12, fmaf(90.0f, i7, 9.0f * i2)))))))))));
      v[14] = fmaf(-4365900.0f, i47, fmaf(1009260.0f, i45, fmaf(-510300.0f, i43, fmaf(-298620.0f, i34, fmaf(84420.0f, i32, fmaf(-28350.0f, i30, fmaf(-23940.0f, i23, fmaf(8820.0f, i21, fmaf(-2340.0f, i14, fmaf(630.0f, i12, fmaf(-300.0f, i7, -30.0f * i2)))))))))));
      v[21] = fmaf(1122660.0f, i34, fmaf(-510300.0f, i32, fmaf(198450.0f, i30, fmaf(90720.0f, i23, fmaf(-50400.0f, i21, fmaf(8820.0f, i14, fmaf(-3150.0f, i12, fmaf(1080.0f, i7, 90.0f * i2))))))));
      v[23] = fmaf(-4252500.0f, i34, fmaf(1009260.0f, i32, fmaf(-311850.0f, i30, fmaf(-292320.0f, i23, fmaf(90720.0f, i21, fmaf(-23940.0f, i14, fmaf(5670.0f, i12, fmaf(-2520.0f, i7, -210.0f * i2))))))));
      v[30] = fmaf(-311850.0f, i23, fmaf(198450.0f, i21, fmaf(-28350.0f, i14, fmaf(11025.0f, i12, fmaf(-3150.0f, i7, -225.0f * i2)))));
      v[32] = fmaf(1009260.0f, i23, fmaf(-510300.0f, i21, fmaf(84420.0f, i14, fmaf(-28350.0f, i12, fmaf(8820.0f, i7, 630.0f * i2)))));
      v[34] = fmaf(-4252500.0f, i23, fmaf(1122660.0f, i21, fmaf(-298620.0f, i14, fmaf(62370.0f, i12, fmaf(-26460.0f, i7, -1890.0f * i2)))));
      v[43] = fmaf(-510300.0f, i14, fmaf(198450.0f, i12, fmaf(-50400.0f, i7, -3150.0f * i2)));
      v[45] = fmaf(1009260.0f, i14, fmaf(-311850.0f, i12, fmaf(90720.0f, i7, 5670.0f * i2)));
      v[47] = fmaf(-4365900.0f, i14, fmaf(810810.0f, i12, fmaf(-332640.0f, i7, -20790.0f * i2)));
      v[56] = fmaf(198450.0f, i7, 11025.0f * i2);
      v[58] = fmaf(-510300.0f, i7, -28350.0f * i2);
      v[60] = fmaf(1122660.0f, i7, 62370.0f * i2);
      v[62] = fmaf(-4864860.0f, i7, -270270.0f * i2);
      v[73] = 198450.0f * i2;
      v[75] = -311850.0f * i2;
      v[77] = 810810.0f * i2;
      v[79] = -4054050.0f * i2;
    }
    {
      const float i5 = v[5]; const float i10 = v[10]; const float i17 = v[17]; const float i19 = v[19]; const float i26 = v[26]; const float i28 = v[28]; const float i37 = v[37]; const float i39 = v[39]; const float i41 = v[41]; const float i50 = v[50]; const float i52 = v[52]; const float i54 = v[54];
      v[5] = fmaf(113400.0f, i54, fmaf(-498960.0f, i52, fmaf(3243240.0f, i50, fmaf(6300.0f, i41, fmaf(-34020.0f, i39, fmaf(207900.0f, i37, fmaf(-2520.0f, i28, fmaf(15120.0f, i26, fmaf(-180.0f, i19, fmaf(1260.0f, i17, fmaf(120.0f, i10, 12.0f * i5)))))))))));
      v[10] = fmaf(113400.0f, i41, fmaf(-612360.0f, i39, fmaf(3742200.0f, i37, fmaf(-40320.0f, i28, fmaf(241920.0f, i26, fmaf(-2520.0f, i19, fmaf(17640.0f, i17, fmaf(1440.0f, i10, 120.0f * i5))))))));
      v[17] = fmaf(-612360.0f, i28, fmaf(3855600.0f, i26, fmaf(-34020.0f, i19, fmaf(248220.0f, i17, fmaf(17640.0f, i10, 1260.0f * i5)))));
      v[19] = fmaf(113400.0f, i28, fmaf(-498960.0f, i26, fmaf(6300.0f, i19, fmaf(-34020.0f, i17, fmaf(-2520.0f, i10, -180.0f * i5)))));
      v[26] = fmaf(-498960.0f, i19, fmaf(3855600.0f, i17, fmaf(241920.0f, i10, 15120.0f * i5)));
      v[28] = fmaf(113400.0f, i19, fmaf(-612360.0f, i17, fmaf(-40320.0f, i10, -2520.0f * i5)));
      v[37] = fmaf(3742200.0f, i10, 207900.0f * i5);
      v[39] = fmaf(-612360.0f, i10, -34020.0f * i5);
      v[41] = fmaf(113400.0f, i10, 6300.0f * i5);
      v[50] = 3243240.0f * i5;
      v[52] = -498960.0f * i5;
      v[54] = 113400.0f * i5;
    }
    v[65] = 0.f; v[67] = 0.f; v[69] = 0.f; v[71] = 0.f; v[81] = 0.f; v[82] = 0.f; v[83] = 0.f; v[84] = 0.f; v[85] = 0.f; v[86] = 0.f; v[87] = 0.f; v[88] = 0.f; v[89] = 0.f; v[90] = 0.f; v[92] = 0.f; v[94] = 0.f; v[96] = 0.f; v[98] = 0.f;
  }
};
template <> struct KFold<10> {
  static constexpr int kNnz = 762;
  static __device__ __forceinline__ void apply(float* v) {
    {
      const float i0 = v[0]; const float i3 = v[3]; const float i6 = v[6]; const float i8 = v[8]; const float i13 = v[13]; const float i15 = v[15]; const float i20 = v[20]; const float i22 = v[22]; const float i24 = v[24]; const float i31 = v[31]; const float i33 = v[33]; const float i35 = v[35]; const float i42 = v[42]; const float i44 = v[44]; const float i46 = v[46]; const float i48 = v[48]; const float i57 = v[57]; const float i59 = v[59]; const float i61 = v[61]; const float i63 = v[63]; const float i72 = v[72]; const float i74 = v[74]; const float i76 = v[76]; const float i78 = v[78]; const float i80 = v[80]; const float i91 = v[91]; const float i93 = v[93]; const float i95 = v[95]; const float i97 = v[97]; const float i99 = v[99]; const float i110 = v[110]; const float i112 = v[112]; const float i114 = v[114]; const float i116 = v[116]; const float i118 = v[118]; const float i120 = v[120];
      v[0] = fmaf(1309458176.0f, i120, fmaf(-68918848.0f, i118, fmaf(12162150.0f, i116, fmaf(-4054050.0f, i114, fmaf(2182950.0f, i112, fmaf(-893025.0f, i110, fmaf(68918848.0f, i99, fmaf(-4054050.0f, i97, fmaf(810810.0f, i95, fmaf(-311850.0f, i93, fmaf(198450.0f, i91, fmaf(4054050.0f, i80, fmaf(-270270.0f, i78, fmaf(62370.0f, i76, fmaf(-28350.0f, i74, fmaf(11025.0f, i72, fmaf(270270.0f, i63, fmaf(-20790.0f, i61, fmaf(5670.0f, i59, fmaf(-3150.0f, i57, fmaf(20790.0f, i48, fmaf(-1890.0f, i46, fmaf(630.0f, i44, fmaf(-225.0f, i42, fmaf(1890.0f, i35, fmaf(-210.0f, i33, fmaf(90.0f, i31, fmaf(210.0f, i24, fmaf(-30.0f, i22, fmaf(9.0f, i20, fmaf(30.0f, i15, fmaf(-6.0f, i13, fmaf(6.0f, i8, 2.0f * i3)))))))))))))))))))))))))))))))));
      v[3] = fmaf(1378376960.0f, i99, fmaf(-81081000.0f, i97, fmaf(16216200.0f, i95, fmaf(-6237000.0f, i93, fmaf(3969000.0f, i91, fmaf(72972896.0f, i80, fmaf(-4864860.0f, i78, fmaf(1122660.0f, i76, fmaf(-510300.0f, i74, fmaf(198450.0f, i72, fmaf(4324320.0f, i63, fmaf(-332640.0f, i61, fmaf(90720.0f, i59, fmaf(-50400.0f, i57, fmaf(291060.0f, i48, fmaf(-26460.0f, i46, fmaf(8820.0f, i44, fmaf(-3150.0f, i42, fmaf(22680.0f, i35, fmaf(-2520.0f, i33, fmaf(1080.0f, i31, fmaf(2100.0f, i24, fmaf(-300.0f, i22, fmaf(90.0f, i20, fmaf(240.0f, i15, fmaf(-48.0f, i13, fmaf(36.0f, i8, fmaf(-6.0f, i6, fmaf(8.0f, i3, 2.0f * i0)))))))))))))))))))))))))))));
      v[6] = fmaf(-68918848.0f, i80, fmaf(12162150.0f, i78, fmaf(-4054050.0f, i76, fmaf(2182950.0f, i74, fmaf(-893025.0f, i72, fmaf(-4054050.0f, i63, fmaf(810810.0f, i61, fmaf(-311850.0f, i59, fmaf(198450.0f, i57, fmaf(-270270.0f, i48, fmaf(62370.0f, i46, fmaf(-28350.0f, i44, fmaf(11025.0f, i42, fmaf(-20790.0f, i35, fmaf(5670.0f, i33, fmaf(-3150.0f, i31, fmaf(-1890.0f, i24, fmaf(630.0f, i22, fmaf(-225.0f, i20, fmaf(-210.0f, i15, fmaf(90.0f, i13, fmaf(-30.0f, i8, fmaf(9.0f, i6, -6.0f * i3)))))))))))))))))))))));
      v[8] = fmaf(1321620352.0f, i80, fmaf(-72972896.0f, i78, fmaf(14345100.0f, i76, fmaf(-5840100.0f, i74, fmaf(2182950.0f, i72, fmaf(69729664.0f, i63, fmaf(-4365900.0f, i61, fmaf(1009260.0f, i59, fmaf(-510300.0f, i57, fmaf(4116420.0f, i48, fmaf(-298620.0f, i46, fmaf(84420.0f, i44, fmaf(-28350.0f, i42, fmaf(275940.0f, i35, fmaf(-23940.0f, i33, fmaf(8820.0f, i31, fmaf(21420.0f, i24, fmaf(-2340.0f, i22, fmaf(630.0f, i20, fmaf(1980.0f, i15, fmaf(-300.0f, i13, fmaf(228.0f, i8, fmaf(-30.0f, i6, fmaf(36.0f, i3, 6.0f * i0))))))))))))))))))))))));
      v[13] = fmaf(-81081000.0f, i63, fmaf(16216200.0f, i61, fmaf(-6237000.0f, i59, fmaf(3969000.0f, i57, fmaf(-4864860.0f, i48, fmaf(1122660.0f, i46, fmaf(-510300.0f, i44, fmaf(198450.0f, i42, fmaf(-332640.0f, i35, fmaf(90720.0f, i33, fmaf(-50400.0f, i31, fmaf(-26460.0f, i24, fmaf(8820.0f, i22, fmaf(-3150.0f, i20, fmaf(-2520.0f, i15, fmaf(1080.0f, i13, fmaf(-300.0f, i8, fmaf(90.0f, i6, fmaf(-48.0f, i3, -6.0f * i0)))))))))))))))))));
      v[15] = fmaf(1313512192.0f, i63, fmaf(-71101800.0f, i61, fmaf(13948200.0f, i59, fmaf(-6237000.0f, i57, fmaf(69230704.0f, i48, fmaf(-4252500.0f, i46, fmaf(1009260.0f, i44, fmaf(-311850.0f, i42, fmaf(4082400.0f, i35, fmaf(-292320.0f, i33, fmaf(90720.0f, i31, fmaf(273420.0f, i24, fmaf(-23940.0f, i22, fmaf(5670.0f, i20, fmaf(21240.0f, i15, fmaf(-2520.0f, i13, fmaf(1980.0f, i8, fmaf(-210.0f, i6, fmaf(240.0f, i3, 30.0f * i0)))))))))))))))))));
      v[20] = fmaf(12162150.0f, i48, fmaf(-4054050.0f, i46, fmaf(2182950.0f, i44, fmaf(-893025.0f, i42, fmaf(810810.0f, i35, fmaf(-311850.0f, i33, fmaf(198450.0f, i31, fmaf(62370.0f, i24, fmaf(-28350.0f, i22, fmaf(11025.0f, i20, fmaf(5670.0f, i15, fmaf(-3150.0f, i13, fmaf(630.0f, i8, fmaf(-225.0f, i6, fmaf(90.0f, i3, 9.0f * i0)))))))))))))));
      v[22] = fmaf(-72972896.0f, i48, fmaf(14345100.0f, i46, fmaf(-5840100.0f, i44, fmaf(2182950.0f, i42, fmaf(-4365900.0f, i35, fmaf(1009260.0f, i33, fmaf(-510300.0f, i31, fmaf(-298620.0f, i24, fmaf(84420.0f, i22, fmaf(-28350.0f, i20, fmaf(-23940.0f, i15, fmaf(8820.0f, i13, fmaf(-2340.0f, i8, fmaf(630.0f, i6, fmaf(-300.0f, i3, -30.0f * i0)))))))))))))));
      v[24] = fmaf(1311641088.0f, i48, fmaf(-70704896.0f, i46, fmaf(14345100.0f, i44, fmaf(-4054050.0f, i42, fmaf(69117296.0f, i35, fmaf(-4252500.0f, i33, fmaf(1122660.0f, i31, fmaf(4076100.0f, i24, fmaf(-298620.0f, i22, fmaf(62370.0f, i20, fmaf(273420.0f, i15, fmaf(-26460.0f, i13, fmaf(21420.0f, i8, fmaf(-1890.0f, i6, fmaf(2100.0f, i3, 210.0f * i0)))))))))))))));
      v[31] = fmaf(16216200.0f, i35, fmaf(-6237000.0f, i33, fmaf(3969000.0f, i31, fmaf(1122660.0f, i24, fmaf(-510300.0f, i22, fmaf(198450.0f, i20, fmaf(90720.0f, i15, fmaf(-50400.0f, i13, fmaf(8820.0f, i8, fmaf(-3150.0f, i6, fmaf(1080.0f, i3, 90.0f * i0)))))))))));
      v[33] = fmaf(-71101800.0f, i35, fmaf(13948200.0f, i33, fmaf(-6237000.0f, i31, fmaf(-4252500.0f, i24, fmaf(1009260.0f, i22, fmaf(-311850.0f, i20, fmaf(-292320.0f, i15, fmaf(90720.0f, i13, fmaf(-23940.0f, i8, fmaf(5670.0f, i6, fmaf(-2520.0f, i3, -210.0f * i0)))))))))));
      v[35] = fmaf(1311244160.0f, i35, fmaf(-71101800.0f, i33, fmaf(16216200.0f, i31, fmaf(69117296.0f, i24, fmaf(-4365900.0f, i22, fmaf(810810.0f, i20, fmaf(4082400.0f, i15, fmaf(-332640.0f, i13, fmaf(275940.0f, i8, fmaf(-20790.0f, i6, fmaf(22680.0f, i3, 1890.0f * i0)))))))))));
      v[42] = fmaf(-4054050.0f, i24, fmaf(2182950.0f, i22, fmaf(-893025.0f, i20, fmaf(-311850.0f, i15, fmaf(198450.0f, i13, fmaf(-28350.0f, i8, fmaf(11025.0f, i6, fmaf(-3150.0f, i3, -225.0f * i0))))))));
      v[44] = fmaf(14345100.0f, i24, fmaf(-5840100.0f, i22, fmaf(2182950.0f, i20, fmaf(1009260.0f, i15, fmaf(-510300.0f, i13, fmaf(84420.0f, i8, fmaf(-28350.0f, i6, fmaf(8820.0f, i3, 630.0f * i0))))))));
      v[46] = fmaf(-70704896.0f, i24, fmaf(14345100.0f, i22, fmaf(-4054050.0f, i20, fmaf(-4252500.0f, i15, fmaf(1122660.0f, i13, fmaf(-298620.0f, i8, fmaf(62370.0f, i6, fmaf(-26460.0f, i3, -1890.0f * i0))))))));
      v[48] = fmaf(1311641088.0f, i24, fmaf(-72972896.0f, i22, fmaf(12162150.0f, i20, fmaf(69230704.0f, i15, fmaf(-4864860.0f, i13, fmaf(4116420.0f, i8, fmaf(-270270.0f, i6, fmaf(291060.0f, i3, 20790.0f * i0))))))));
      v[57] = fmaf(-6237000.0f, i15, fmaf(3969000.0f, i13, fmaf(-510300.0f, i8, fmaf(198450.0f, i6, fmaf(-50400.0f, i3, -3150.0f * i0)))));
      v[59] = fmaf(13948200.0f, i15, fmaf(-6237000.0f, i13, fmaf(1009260.0f, i8, fmaf(-311850.0f, i6, fmaf(90720.0f, i3, 5670.0f * i0)))));
      v[61] = fmaf(-71101800.0f, i15, fmaf(16216200.0f, i13, fmaf(-4365900.0f, i8, fmaf(810810.0f, i6, fmaf(-332640.0f, i3, -20790.0f * i0)))));
      v[63] = fmaf(1313512192.0f, i15, fmaf(-81081000.0f, i13, fmaf(69729664.0f, i8, fmaf(-4054050.0f, i6, fmaf(4324320.0f, i3, 270270.0f * i0)))));
      v[72] = fmaf(2182950.0f, i8, fmaf(-893025.0f, i6, fmaf(198450.0f, i3, 11025.0f * i0)));
      v[74] = fmaf(-5840100.0f, i8, fmaf(2182950.0f, i6, fmaf(-510300.0f, i3, -28350.0f * i0)));
      v[76] = fmaf(14345100.0f, i8, fmaf(-4054050.0f, i6, fmaf(1122660.0f, i3, 62370.0f * i0)));
      v[78] = fmaf(-72972896.0f, i8, fmaf(12162150.0f, i6, fmaf(-4864860.0f, i3, -270270.0f * i0)));
      v[80] = fmaf(1321620352.0f, i8, fmaf(-68918848.0f, i6, fmaf(72972896.0f, i3, 4054050.0f * i0)));
      v[91] = fmaf(3969000.0f, i3, 198450.0f * i0);
      v[93] = fmaf(-6237000.0f, i3, -311850.0f * i0);
      v[95] = fmaf(16216200.0f, i3, 810810.0f * i0);
      v[97] = fmaf(-81081000.0f, i3, -4054050.0f * i0);
      v[99] = fmaf(1378376960.0f, i3, 68918848.0f * i0);
      v[110] = -893025.0f * i0;
      v[112] = 2182950.0f * i0;
      v[114] = -4054050.0f * i0;
      v[116] = 12162150.0f * i0;
      v[118] = -68918848.0f * i0;
      v[120] = 1309458176.0f * i0;
    }
    {
      const float i1 = v[1]; const float i4 = v[4]; const float i9 = v[9]; const float i11 = v[11]; const float i16 = v[16]; const float i18 = v[18]; const float i25 = v[25]; const float i27 = v[27]; const float i29 = v[29]; const float i36 = v[36]; const float i38 = v[38]; const float i40 = v[40]; const float i49 = v[49]; const float i51 = v[51]; const float i53 = v[53]; const float i55 = v[55]; const float i64 = v[64]; const float i66 = v[66]; const float i68 = v[68]; const float i70 = v[70]; const float i81 = v[81]; const float i83 = v[83]; const float i85 = v[85]; const float i87 = v[87]; const float i89 = v[89];
      v[1] = fmaf(-396900.0f, i89, fmaf(1871100.0f, i87, fmaf(-8108100.0f, i85, fmaf(56756700.0f, i83, fmaf(-1240539264.0f, i81, fmaf(113400.0f, i70, fmaf(-498960.0f, i68, fmaf(3243240.0f, i66, fmaf(-64864800.0f, i64, fmaf(6300.0f, i55, fmaf(-34020.0f, i53, fmaf(207900.0f, i51, fmaf(-3783780.0f, i49, fmaf(-2520.0f, i40, fmaf(15120.0f, i38, fmaf(-249480.0f, i36, fmaf(-180.0f, i29, fmaf(1260.0f, i27, fmaf(-18900.0f, i25, fmaf(120.0f, i18, fmaf(-1680.0f, i16, fmaf(12.0f, i11, fmaf(-180.0f, i9, fmaf(-24.0f, i4, -4.0f * i1))))))))))))))))))))))));
      v[4] = fmaf(2268000.0f, i70, fmaf(-9979200.0f, i68, fmaf(64864800.0f, i66, fmaf(-1297296000.0f, i64, fmaf(113400.0f, i55, fmaf(-612360.0f, i53, fmaf(3742200.0f, i51, fmaf(-68108040.0f, i49, fmaf(-40320.0f, i40, fmaf(241920.0f, i38, fmaf(-3991680.0f, i36, fmaf(-2520.0f, i29, fmaf(17640.0f, i27, fmaf(-264600.0f, i25, fmaf(1440.0f, i18, fmaf(-20160.0f, i16, fmaf(120.0f, i11, fmaf(-1800.0f, i9, fmaf(-192.0f, i4, -24.0f * i1)))))))))))))))))));
      v[9] = fmaf(1871100.0f, i55, fmaf(-10376100.0f, i53, fmaf(66735900.0f, i51, fmaf(-1305404160.0f, i49, fmaf(-612360.0f, i40, fmaf(3855600.0f, i38, fmaf(-68607000.0f, i36, fmaf(-34020.0f, i29, fmaf(248220.0f, i27, fmaf(-4025700.0f, i25, fmaf(17640.0f, i18, fmaf(-267120.0f, i16, fmaf(1260.0f, i11, fmaf(-20340.0f, i9, fmaf(-1800.0f, i4, -180.0f * i1)))))))))))))));
      v[11] = fmaf(-396900.0f, i55, fmaf(1871100.0f, i53, fmaf(-8108100.0f, i51, fmaf(56756700.0f, i49, fmaf(113400.0f, i40, fmaf(-498960.0f, i38, fmaf(3243240.0f, i36, fmaf(6300.0f, i29, fmaf(-34020.0f, i27, fmaf(207900.0f, i25, fmaf(-2520.0f, i18, fmaf(15120.0f, i16, fmaf(-180.0f, i11, fmaf(1260.0f, i9, fmaf(120.0f, i4, 12.0f * i1)))))))))))))));
      v[16] = fmaf(-9979200.0f, i40, fmaf(67132800.0f, i38, fmaf(-1307275264.0f, i36, fmaf(-498960.0f, i29, fmaf(3855600.0f, i27, fmaf(-68720400.0f, i25, fmaf(241920.0f, i18, fmaf(-4032000.0f, i16, fmaf(15120.0f, i11, fmaf(-267120.0f, i9, fmaf(-20160.0f, i4, -1680.0f * i1)))))))))));
      v[18] = fmaf(2268000.0f, i40, fmaf(-9979200.0f, i38, fmaf(64864800.0f, i36, fmaf(113400.0f, i29, fmaf(-612360.0f, i27, fmaf(3742200.0f, i25, fmaf(-40320.0f, i18, fmaf(241920.0f, i16, fmaf(-2520.0f, i11, fmaf(17640.0f, i9, fmaf(1440.0f, i4, 120.0f * i1)))))))))));
      v[25] = fmaf(-8108100.0f, i29, fmaf(66735900.0f, i27, fmaf(-1307672064.0f, i25, fmaf(3742200.0f, i18, fmaf(-68720400.0f, i16, fmaf(207900.0f, i11, fmaf(-4025700.0f, i9, fmaf(-264600.0f, i4, -18900.0f * i1))))))));
      v[27] = fmaf(1871100.0f, i29, fmaf(-10376100.0f, i27, fmaf(66735900.0f, i25, fmaf(-612360.0f, i18, fmaf(3855600.0f, i16, fmaf(-34020.0f, i11, fmaf(248220.0f, i9, fmaf(17640.0f, i4, 1260.0f * i1))))))));
      v[29] = fmaf(-396900.0f, i29, fmaf(1871100.0f, i27, fmaf(-8108100.0f, i25, fmaf(113400.0f, i18, fmaf(-498960.0f, i16, fmaf(6300.0f, i11, fmaf(-34020.0f, i9, fmaf(-2520.0f, i4, -180.0f * i1))))))));
      v[36] = fmaf(64864800.0f, i18, fmaf(-1307275264.0f, i16, fmaf(3243240.0f, i11, fmaf(-68607000.0f, i9, fmaf(-3991680.0f, i4, -249480.0f * i1)))));
      v[38] = fmaf(-9979200.0f, i18, fmaf(67132800.0f, i16, fmaf(-498960.0f, i11, fmaf(3855600.0f, i9, fmaf(241920.0f, i4, 15120.0f * i1)))));
      v[40] = fmaf(2268000.0f, i18, fmaf(-9979200.0f, i16, fmaf(113400.0f, i11, fmaf(-612360.0f, i9, fmaf(-40320.0f, i4, -2520.0f * i1)))));
      v[49] = fmaf(56756700.0f, i11, fmaf(-1305404160.0f, i9, fmaf(-68108040.0f, i4, -3783780.0f * i1)));
      v[51] = fmaf(-8108100.0f, i11, fmaf(66735900.0f, i9, fmaf(3742200.0f, i4, 207900.0f * i1)));
      v[53] = fmaf(1871100.0f, i11, fmaf(-10376100.0f, i9, fmaf(-612360.0f, i4, -34020.0f * i1)));
      v[55] = fmaf(-396900.0f, i11, fmaf(1871100.0f, i9, fmaf(113400.0f, i4, 6300.0f * i1)));
      v[64] = fmaf(-1297296000.0f, i4, -64864800.0f * i1);
      v[66] = fmaf(64864800.0f, i4, 3243240.0f * i1);
      v[68] = fmaf(-9979200.0f, i4, -498960.0f * i1);
      v[70] = fmaf(2268000.0f, i4, 113400.0f * i1);
      v[81] = -1240539264.0f * i1;
      v[83] = 56756700.0f * i1;
      v[85] = -8108100.0f * i1;
      v[87] = 1871100.0f * i1;
      v[89] = -396900.0f * i1;
    }
    {
      const float i2 = v[2]; const float i7 = v[7]; const float i12 = v[12]; const float i14 = v[14]; const float i21 = v[21]; const float i23 = v[23]; const float i30 = v[30]; const float i32 = v[32]; const float i34 = v[34]; const float i43 = v[43]; const float i45 = v[45]; const float i47 = v[47]; const float i56 = v[56]; const float i58 = v[58]; const float i60 = v[60]; const float i62 = v[62]; const float i73 = v[73]; const float i75 = v[75]; const float i77 = v[77]; const float i79 = v[79]; const float i90 = v[90]; const float i92 = v[92]; const float i94 = v[94]; const float i96 = v[96]; const float i98 = v[98];
      v[2] = fmaf(-68918848.0f, i98, fmaf(12162150.0f, i96, fmaf(-4054050.0f, i94, fmaf(2182950.0f, i92, fmaf(-893025.0f, i90, fmaf(-4054050.0f, i79, fmaf(810810.0f, i77, fmaf(-311850.0f, i75, fmaf(198450.0f, i73, fmaf(-270270.0f, i62, fmaf(62370.0f, i60, fmaf(-28350.0f, i58, fmaf(11025.0f, i56, fmaf(-20790.0f, i47, fmaf(5670.0f, i45, fmaf(-3150.0f, i43, fmaf(-1890.0f, i34, fmaf(630.0f, i32, fmaf(-225.0f, i30, fmaf(-210.0f, i23, fmaf(90.0f, i21, fmaf(-30.0f, i14, fmaf(9.0f, i12, -6.0f * i7)))))))))))))))))))))));
      v[7] = fmaf(-81081000.0f, i79, fmaf(16216200.0f, i77, fmaf(-6237000.0f, i75, fmaf(3969000.0f, i73, fmaf(-4864860.0f, i62, fmaf(1122660.0f, i60, fmaf(-510300.0f, i58, fmaf(198450.0f, i56, fmaf(-332640.0f, i47, fmaf(90720.0f, i45, fmaf(-50400.0f, i43, fmaf(-26460.0f, i34, fmaf(8820.0f, i32, fmaf(-3150.0f, i30, fmaf(-2520.0f, i23, fmaf(1080.0f, i21, fmaf(-300.0f, i14, fmaf(90.0f, i12, fmaf(-48.0f, i7, -6.0f * i2)))))))))))))))))));
      v[12] = fmaf(12162150.0f, i62, fmaf(-4054050.0f, i60, fmaf(2182950.0f, i58, fmaf(-893025.0f, i56, fmaf(810810.0f, i47, fmaf(-311850.0f, i45, fmaf(198450.0f, i43, fmaf(62370.0f, i34, fmaf(-28350.0f, i32, fmaf(11025.0f, i30, fmaf(5670.0f, i23, fmaf(-3150.0f, i21, fmaf(630.0f, i14, fmaf(-225.0f, i12, fmaf(90.0f, i7, 9.0f * i2)))))))))))))));
      v[14] = fmaf(-72972896.0f, i62, fmaf(14345100.0f, i60, fmaf(-5840100.0f, i58, fmaf(2182950.0f, i56, fmaf(-4365900.0f, i47, fmaf(1009260.0f, i45, fmaf(-510300.0f, i43, fmaf(-298620.0f, i34, fmaf(84420.0f, i32, fmaf(-28350.0f, i30, fmaf(-23940.0f, i23, fmaf(8820.0f, i21, fmaf(-2340.0f, i14, fmaf(630.0f, i12, fmaf(-300.0f, i7, -30.0f * i2)))))))))))))));
      v[21] = fmaf(16216200.0f, i47, fmaf(-6237000.0f, i45, fmaf(3969000.0f, i43, fmaf(1122660.0f, i34, fmaf(-510300.0f, i32, fmaf(198450.0f, i30, fmaf(90720.0f, i23, fmaf(-50400.0f, i21, fmaf(8820.0f, i14, fmaf(-3150.0f, i12, fmaf(1080.0f, i7, 90.0f * i2)))))))))));
      v[23] = fmaf(-71101800.0f, i47, fmaf(13948200.0f, i45, fmaf(-6237000.0f, i43, fmaf(-4252500.0f, i34, fmaf(1009260.0f, i32, fmaf(-311850.0f, i30, fmaf(-292320.0f, i23, fmaf(90720.0f, i21, fmaf(-23940.0f, i14, fmaf(5670.0f, i12, fmaf(-2520.0f, i7, -210.0f * i2)))))))))));
      v[30] = fmaf(-4054050.0f, i34, fmaf(2182950.0f, i32, fmaf(-893025.0f, i30, fmaf(-311850.0f, i23, fmaf(198450.0f, i21, fmaf(-28350.0f, i14, fmaf(11025.0f, i12, fmaf(-3150.0f, i7, -225.0f * i2))))))));
      v[32] = fmaf(14345100.0f, i34, fmaf(-5840100.0f, i32, fmaf(2182950.0f, i30, fmaf(1009260.0f, i23, fmaf(-510300.0f, i21, fmaf(84420.0f, i14, fmaf(-28350.0f, i12, fmaf(8820.0f, i7, 630.0f * i2))))))));
      v[34] = fmaf(-70704896.0f, i34, fmaf(14345100.0f, i32, fmaf(-4054050.0f, i30, fmaf(-4252500.0f, i23, fmaf(1122660.0f, i21, fmaf(-298620.0f, i14, fmaf(62370.0f, i12, fmaf(-26460.0f, i7, -1890.0f * i2))))))));
      v[43] = fmaf(-6237000.0f, i23, fmaf(3969000.0f, i21, fmaf(-510300.0f, i14, fmaf(198450.0f, i12, fmaf(-50400.0f, i7, -3150.0f * i2)))));
      v[45] = fmaf(13948200.0f, i23, fmaf(-6237000.0f, i21, fmaf(1009260.0f, i14, fmaf(-311850.0f, i12, fmaf(90720.0f, i7, 5670.0f * i2)))));
      v[47] = fmaf(-71101800.0f, i23, fmaf(16216200.0f, i21, fmaf(-4365900.0f, i14, fmaf(810810.0f, i12, fmaf(-332640.0f, i7, -20790.0f * i2)))));
      v[56] = fmaf(2182950.0f, i14, fmaf(-893025.0f, i12, fmaf(198450.0f, i7, 11025.0f * i2)));
      v[58] = fmaf(-5840100.0f, i14, fmaf(2182950.0f, i12, fmaf(-510300.0f, i7, -28350.0f * i2)));
      v[60] = fmaf(14345100.0f, i14, fmaf(-4054050.0f, i12, fmaf(1122660.0f, i7, 62370.0f * i2)));
      v[62] = fmaf(-72972896.0f, i14, fmaf(12162150.0f, i12, fmaf(-4864860.0f, i7, -270270.0f * i2)));
      v[73] = fmaf(3969000.0f, i7, 198450.0f * i2);
      v[75] = fmaf(-6237000.0f, i7, -311850.0f * i2);
      v[77] = fmaf(16216200.0f, i7, 810810.0f * i2);
      v[79] = fmaf(-81081000.0f, i7, -4054050.0f * i2);
      v[90] = -893025.0f * i2;
      v[92] = 2182950.0f * i2;
      v[94] = -4054050.0f * i2;
      v[96] = 12162150.0f * i2;
      v[98] = -68918848.0f * i2;
    }
    {
      const float i5 = v[5]; const float i10 = v[10]; const float i17 = v[17]; const float i19 = v[19]; const float i26 = v[26]; const float i28 = v[28]; const float i37 = v[37]; const float i39 = v[39]; const float i41 = v[41]; const float i50 = v[50]; const float i52 = v[52]; const float i54 = v[54]; const float i65 = v[65]; const float i67 = v[67]; const float i69 = v[69]; const float i71 = v[71];
      v[5] = fmaf(-396900.0f, i71, fmaf(1871100.0f, i69, fmaf(-8108100.0f, i67, fmaf(56756700.0f, i65, fmaf(113400.0f, i54, fmaf(-498960.0f, i52, fmaf(3243240.0f, i50, fmaf(6300.0f, i41, fmaf(-34020.0f, i39, fmaf(207900.0f, i37, fmaf(-2520.0f, i28, fmaf(15120.0f, i26, fmaf(-180.0f, i19, fmaf(1260.0f, i17, fmaf(120.0f, i10, 12.0f * i5)))))))))))))));
      v[10] = fmaf(2268000.0f, i54, fmaf(-9979200.0f, i52, fmaf(64864800.0f, i50, fmaf(113400.0f, i41, fmaf(-612360.0f, i39, fmaf(3742200.0f, i37, fmaf(-40320.0f, i28, fmaf(241920.0f, i26, fmaf(-2520.0f, i19, fmaf(17640.0f, i17, fmaf(1440.0f, i10, 120.0f * i5)))))))))));
      v[17] = fmaf(1871100.0f, i41, fmaf(-10376100.0f, i39, fmaf(66735900.0f, i37, fmaf(-612360.0f, i28, fmaf(3855600.0f, i26, fmaf(-34020.0f, i19, fmaf(248220.0f, i17, fmaf(17640.0f, i10, 1260.0f * i5))))))));
      v[19] = fmaf(-396900.0f, i41, fmaf(1871100.0f, i39, fmaf(-8108100.0f, i37, fmaf(113400.0f, i28, fmaf(-498960.0f, i26, fmaf(6300.0f, i19, fmaf(-34020.0f, i17, fmaf(-2520.0f, i10, -180.0f * i5))))))));
      v[26] = fmaf(-9979200.0f, i28, fmaf(67132800.0f, i26, fmaf(-498960.0f, i19, fmaf(3855600.0f, i17, fmaf(241920.0f, i10, 15120.0f * i5)))));
      v[28] = fmaf(2268000.0f, i28, fmaf(-9979200.0f, i26, fmaf(113400.0f, i19, fmaf(-612360.0f, i17, fmaf(-40320.0f, i10, -2520.0f * i5)))));
      v[37] = fmaf(-8108100.0f, i19, fmaf(66735900.0f, i17, fmaf(3742200.0f, i10, 207900.0f * i5)));
      v[39] = fmaf(1871100.0f, i19, fmaf(-10376100.0f, i17, fmaf(-612360.0f, i10, -34020.0f * i5)));
      v[41] = fmaf(-396900.0f, i19, fmaf(1871100.0f, i17, fmaf(113400.0f, i10, 6300.0f * i5)));
      v[50] = fmaf(64864800.0f, i10, 3243240.0f * i5);
      v[52] = fmaf(-9979200.0f, i10, -498960.0f * i5);
      v[54] = fmaf(2268000.0f, i10, 113400.0f * i5);
      v[65] = 56756700.0f * i5;
      v[67] = -8108100.0f * i5;
      v[69] = 1871100.0f * i5;
      v[71] = -396900.0f * i5;
    }
    v[82] = 0.f; v[84] = 0.f; v[86] = 0.f; v[88] = 0.f; v[100] = 0.f; v[101] = 0.f; v[102] = 0.f; v[103] = 0.f; v[104] = 0.f; v[105] = 0.f; v[106] = 0.f; v[107] = 0.f; v[108] = 0.f; v[109] = 0.f; v[111] = 0.f; v[113] = 0.f; v[115] = 0.f; v[117] = 0.f; v[119] = 0.f;
  }
};
}  // namespace jb
