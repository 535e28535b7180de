// Constant tables of the engine: ITU-T H.264 scales and scans, and the x264-derived constants of
// ragdoll's Balanced preset. Values equal the reference's (the bitstream depends on them):
//   crates/ragdoll-codec/src/h264/enc.rs:64-98   lambda per QP, decimation weights
//   crates/ragdoll-codec/src/h264.rs:1174-1370   zig-zag scans, (de)quantisation scales, chroma QP
//   crates/ragdoll-simd/src/h264_dsp.rs:16-110   deblocking alpha / beta / tc0
#pragma once
#include <cstdint>

namespace rg {
namespace tables {

// x264 lambda of the SAD/SATD domain, QP 0..51.
inline constexpr uint16_t kLambda[52] = {1,  1,  1,  1,  1,  1,  1,  1,  1,  1,  1,  1,  1,
                                         1,  1,  1,  2,  2,  2,  2,  3,  3,  3,  4,  4,  4,
                                         5,  6,  6,  7,  8,  9,  10, 11, 13, 14, 16, 18, 20,
                                         23, 25, 29, 32, 36, 40, 45, 51, 57, 64, 72, 81, 91};
// Decimation weight by the zero run before a +-1 level (4x4 and 8x8 blocks).
inline constexpr uint8_t kDecimate4[16] = {3, 2, 2, 1, 1, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
inline constexpr uint8_t kDecimate8[64] = {3, 3, 3, 3, 2, 2, 2, 2, 2, 2, 2, 2, 1, 1, 1, 1,
                                           1, 1, 1, 1, 1, 1, 1, 1};  // rest 0
// Frame zig-zag scans (Tables 8-12, 8-13): scan position -> raster position.
inline constexpr uint8_t kScan4[16] = {0, 1, 4, 8, 5, 2, 3, 6, 9, 12, 13, 10, 7, 11, 14, 15};
inline constexpr uint8_t kScan8[64] = {
    0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,  12, 19, 26, 33, 40, 48,
    41, 34, 27, 20, 13, 6,  7,  14, 21, 28, 35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23,
    30, 37, 44, 51, 58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};
// Quantiser multipliers MF and dequantiser scales by QP%6, per position class.
inline constexpr uint16_t kMf4[6][3] = {{13107, 5243, 8066}, {11916, 4660, 7490}, {10082, 4194, 6554},
                                        {9362, 3647, 5825},  {8192, 3355, 5243},  {7282, 2893, 4559}};
inline constexpr uint8_t kDq4[6][3] = {{10, 16, 13}, {11, 18, 14}, {13, 20, 16},
                                       {14, 23, 18}, {16, 25, 20}, {18, 29, 23}};
inline constexpr uint16_t kMf8[6][6] = {{13107, 11428, 20972, 12222, 16777, 15481},
                                        {11916, 10826, 19174, 11058, 14980, 14290},
                                        {10082, 8943, 15978, 9675, 12710, 11985},
                                        {9362, 8228, 14913, 8931, 11984, 11259},
                                        {8192, 7346, 13159, 7740, 10486, 9777},
                                        {7282, 6428, 11570, 6830, 9118, 8640}};
inline constexpr uint8_t kDq8[6][6] = {{20, 18, 32, 19, 25, 24}, {22, 19, 35, 21, 28, 26},
                                       {26, 23, 42, 24, 33, 31}, {28, 25, 45, 26, 35, 33},
                                       {32, 28, 51, 30, 40, 38}, {36, 32, 58, 34, 46, 43}};
// QP_Y -> QP_C (Table 8-15).
inline constexpr uint8_t kChromaQp[52] = {0,  1,  2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12,
                                          13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 25,
                                          26, 27, 28, 29, 29, 30, 31, 32, 32, 33, 34, 34, 35,
                                          35, 36, 36, 37, 37, 37, 38, 38, 38, 39, 39, 39, 39};
// Deblocking thresholds by indexA / indexB (Table 8-16) and tC0 (Table 8-17), bS 1..3.
inline constexpr uint8_t kAlpha[52] = {0,  0,  0,  0,  0,  0,  0,   0,   0,   0,   0,   0,   0,
                                       0,  0,  0,  4,  4,  5,  6,   7,   8,   9,   10,  12,  13,
                                       15, 17, 20, 22, 25, 28, 32,  36,  40,  45,  50,  56,  63,
                                       71, 80, 90, 101, 113, 127, 144, 162, 182, 203, 226, 255, 255};
inline constexpr uint8_t kBeta[52] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0,  0,  0,  0,  0,  0,  0,  2,  2,
                                      2, 3, 3, 3, 3, 4, 4, 4, 6, 6,  7,  7,  8,  8,  9,  9,  10, 10,
                                      11, 11, 12, 12, 13, 13, 14, 14, 15, 15, 16, 16, 17, 17, 18, 18};
inline constexpr uint8_t kTc0[52][3] = {
    {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0},  {0, 0, 0},  {0, 0, 0},   {0, 0, 0},
    {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0},  {0, 0, 0},  {0, 0, 0},   {0, 0, 0},
    {0, 0, 0}, {0, 0, 1}, {0, 0, 1}, {0, 0, 1}, {0, 0, 1},  {0, 1, 1},  {0, 1, 1},   {1, 1, 1},
    {1, 1, 1}, {1, 1, 1}, {1, 1, 1}, {1, 1, 2}, {1, 1, 2},  {1, 1, 2},  {1, 1, 2},   {1, 2, 3},
    {1, 2, 3}, {2, 2, 3}, {2, 2, 4}, {2, 3, 4}, {2, 3, 4},  {3, 3, 5},  {3, 4, 6},   {3, 4, 6},
    {4, 5, 7}, {4, 5, 8}, {4, 6, 9}, {5, 7, 10}, {6, 8, 11}, {6, 8, 13}, {7, 10, 14}, {8, 11, 16},
    {9, 12, 18}, {10, 13, 20}, {11, 15, 23}, {13, 17, 25}};

}  // namespace tables
}  // namespace rg
