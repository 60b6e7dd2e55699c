// Tile shapes of the fused kernel compiled per K and state width (rows x
// slices x slices per thread; W = 4 for FP32, 2 for the 16-bit formats); the
// first entry is the default of the exact arithmetic, entry `fast` the
// default of the fast one (K = 3, FP32: 8 x 128 x 4 measured 3 % faster than
// 16 x 64 x 2 at 768^2 x 1024).  Each shape is compiled in the exact and the
// fast arithmetic (fused_*.cu).
#pragma once

namespace potts {

template <int K, int W>
struct TileShapes;
template <int W> struct TileShapes<2, W> { static constexpr int n = 2, fast = 0; static constexpr int r[n] = {8, 8}, t[n] = {128, 64}, v[n] = {2, 4}; };
template <> struct TileShapes<3, 4> { static constexpr int n = 4, fast = 3; static constexpr int r[n] = {16, 8, 8, 8}, t[n] = {64, 128, 64, 128}, v[n] = {2, 2, 2, 4}; };
template <> struct TileShapes<3, 2> { static constexpr int n = 2, fast = 0; static constexpr int r[n] = {16, 8}, t[n] = {64, 128}, v[n] = {2, 2}; };
template <> struct TileShapes<4, 4> { static constexpr int n = 3, fast = 0; static constexpr int r[n] = {8, 8, 4}, t[n] = {64, 64, 128}, v[n] = {2, 4, 4}; };
template <> struct TileShapes<4, 2> { static constexpr int n = 1, fast = 0; static constexpr int r[n] = {8}, t[n] = {64}, v[n] = {2}; };
template <int W> struct TileShapes<5, W> { static constexpr int n = 2, fast = 0; static constexpr int r[n] = {4, 8}, t[n] = {64, 64}, v[n] = {4, 2}; };
template <> struct TileShapes<6, 4> { static constexpr int n = 1, fast = 0; static constexpr int r[n] = {4}, t[n] = {64}, v[n] = {4}; };
template <> struct TileShapes<6, 2> { static constexpr int n = 2, fast = 0; static constexpr int r[n] = {4, 8}, t[n] = {64, 64}, v[n] = {4, 2}; };

template <int K, typename ST>
using ShapesOf = TileShapes<K, (int)sizeof(ST) == 4 ? 4 : 2>;

}  // namespace potts
