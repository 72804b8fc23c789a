// Generated by gen_stencils.py -- do not edit.
// Exact dyadic 1-D prolongation weights (see gen_stencils.py for the
// derivation); every value is exactly representable in FP64.
#pragma once
#if defined(__CUDACC__)
#define CXB_HD __host__ __device__
#else
#define CXB_HD
#endif
namespace cxb {
CXB_HD constexpr double kVcPoly1(int i) { return i == 0 ? 1.0 / 2.0 : i == 1 ? 1.0 / 2.0 : 0.0; }
constexpr int kVcPoly1Len = 2;
CXB_HD constexpr double kVcPoly3(int i) { return i == 0 ? -1.0 / 16.0 : i == 1 ? 9.0 / 16.0 : i == 2 ? 9.0 / 16.0 : i == 3 ? -1.0 / 16.0 : 0.0; }
constexpr int kVcPoly3Len = 4;
CXB_HD constexpr double kVcPoly5(int i) { return i == 0 ? 3.0 / 256.0 : i == 1 ? -25.0 / 256.0 : i == 2 ? 75.0 / 128.0 : i == 3 ? 75.0 / 128.0 : i == 4 ? -25.0 / 256.0 : i == 5 ? 3.0 / 256.0 : 0.0; }
constexpr int kVcPoly5Len = 6;
CXB_HD constexpr double kVcPoly7(int i) { return i == 0 ? -5.0 / 2048.0 : i == 1 ? 49.0 / 2048.0 : i == 2 ? -245.0 / 2048.0 : i == 3 ? 1225.0 / 2048.0 : i == 4 ? 1225.0 / 2048.0 : i == 5 ? -245.0 / 2048.0 : i == 6 ? 49.0 / 2048.0 : i == 7 ? -5.0 / 2048.0 : 0.0; }
constexpr int kVcPoly7Len = 8;
CXB_HD constexpr double kCcPoly1(int i) { return i == 0 ? 1.0 / 4.0 : i == 1 ? 3.0 / 4.0 : 0.0; }
constexpr int kCcPoly1Len = 2;
CXB_HD constexpr double kCcPoly3(int i) { return i == 0 ? -5.0 / 128.0 : i == 1 ? 35.0 / 128.0 : i == 2 ? 105.0 / 128.0 : i == 3 ? -7.0 / 128.0 : 0.0; }
constexpr int kCcPoly3Len = 4;
CXB_HD constexpr double kCcPoly5(int i) { return i == 0 ? 63.0 / 8192.0 : i == 1 ? -495.0 / 8192.0 : i == 2 ? 1155.0 / 4096.0 : i == 3 ? 3465.0 / 4096.0 : i == 4 ? -693.0 / 8192.0 : i == 5 ? 77.0 / 8192.0 : 0.0; }
constexpr int kCcPoly5Len = 6;
CXB_HD constexpr double kCcPoly7(int i) { return i == 0 ? -429.0 / 262144.0 : i == 1 ? 4095.0 / 262144.0 : i == 2 ? -19305.0 / 262144.0 : i == 3 ? 75075.0 / 262144.0 : i == 4 ? 225225.0 / 262144.0 : i == 5 ? -27027.0 / 262144.0 : i == 6 ? 5005.0 / 262144.0 : i == 7 ? -495.0 / 262144.0 : 0.0; }
constexpr int kCcPoly7Len = 8;
CXB_HD constexpr double kCcCons0(int i) { return i == 0 ? 1.0 / 1.0 : 0.0; }
constexpr int kCcCons0Len = 1;
CXB_HD constexpr double kCcCons1(int i) { return i == 0 ? 1.0 / 4.0 : i == 1 ? 3.0 / 4.0 : 0.0; }
constexpr int kCcCons1Len = 2;
CXB_HD constexpr double kCcCons2(int i) { return i == 0 ? 1.0 / 8.0 : i == 1 ? 1.0 / 1.0 : i == 2 ? -1.0 / 8.0 : 0.0; }
constexpr int kCcCons2Len = 3;
CXB_HD constexpr double kCcCons3(int i) { return i == 0 ? -3.0 / 64.0 : i == 1 ? 17.0 / 64.0 : i == 2 ? 55.0 / 64.0 : i == 3 ? -5.0 / 64.0 : 0.0; }
constexpr int kCcCons3Len = 4;
CXB_HD constexpr double kCcCons4(int i) { return i == 0 ? -3.0 / 128.0 : i == 1 ? 11.0 / 64.0 : i == 2 ? 1.0 / 1.0 : i == 3 ? -11.0 / 64.0 : i == 4 ? 3.0 / 128.0 : 0.0; }
constexpr int kCcCons4Len = 5;
CXB_HD constexpr double kCcCons5(int i) { return i == 0 ? 5.0 / 512.0 : i == 1 ? -37.0 / 512.0 : i == 2 ? 69.0 / 256.0 : i == 3 ? 231.0 / 256.0 : i == 4 ? -63.0 / 512.0 : i == 5 ? 7.0 / 512.0 : 0.0; }
constexpr int kCcCons5Len = 6;
CXB_HD constexpr double kCcCons6(int i) { return i == 0 ? 5.0 / 1024.0 : i == 1 ? -11.0 / 256.0 : i == 2 ? 201.0 / 1024.0 : i == 3 ? 1.0 / 1.0 : i == 4 ? -201.0 / 1024.0 : i == 5 ? 11.0 / 256.0 : i == 6 ? -5.0 / 1024.0 : 0.0; }
constexpr int kCcCons6Len = 7;
CXB_HD constexpr double kCcCons7(int i) { return i == 0 ? -35.0 / 16384.0 : i == 1 ? 325.0 / 16384.0 : i == 2 ? -1439.0 / 16384.0 : i == 3 ? 4441.0 / 16384.0 : i == 4 ? 15159.0 / 16384.0 : i == 5 ? -2481.0 / 16384.0 : i == 6 ? 459.0 / 16384.0 : i == 7 ? -45.0 / 16384.0 : 0.0; }
constexpr int kCcCons7Len = 8;
CXB_HD constexpr double kCcEno2Row0(int i) { return i == 0 ? -1.0 / 8.0 : i == 1 ? 1.0 / 2.0 : i == 2 ? 5.0 / 8.0 : 0.0; }
constexpr int kCcEno2Row0Len = 3;
CXB_HD constexpr double kCcEno2Row1(int i) { return i == 0 ? 1.0 / 8.0 : i == 1 ? 1.0 / 1.0 : i == 2 ? -1.0 / 8.0 : 0.0; }
constexpr int kCcEno2Row1Len = 3;
CXB_HD constexpr double kCcEno2Row2(int i) { return i == 0 ? 11.0 / 8.0 : i == 1 ? -1.0 / 2.0 : i == 2 ? 1.0 / 8.0 : 0.0; }
constexpr int kCcEno2Row2Len = 3;
}  // namespace cxb
