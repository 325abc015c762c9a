// Host-side geometry of the dense stage: plane list, flow matrices, skip masks, approximate reciprocals.
// These run once per layer on a handful of values; the per-pixel work is on the GPU.
#pragma once
#include <cstdint>
#include <vector>

#include "../../include/lux_sgm.h"

namespace lux {

uint32_t host_rcp_bits(uint32_t b);    // IntelApprox.RcpBits (Lux.Engine/Imaging/IntelApprox.cs:21-29)
uint32_t host_rsqrt_bits(uint32_t b);  // IntelApprox.RsqrtBits (IntelApprox.cs:32-45)
float host_rcp(float x);
const uint32_t* host_rcp_table();      // the 4096-entry table (uploaded to the device once per context)

// DenseStereo.Planes (DenseStereo.cs:41-88); returns a LUX_ERR_* code.
int host_planes(float near_, float far_, const lux_calib* calibs, int ncams, float density, int align, std::vector<float>& out);
// Mat4D.FlowMatrix (ViewTransform.cs:126-133): column-major float M = (K_b·E_b)·(K_a·E_a)^-1 computed in double.
void host_flow_matrix(const lux_calib& a, const lux_calib& b, float out[16]);
// DenseLayer.SkipMask (DenseStereoSgm.cs:65-87) seeds a fresh generator for every 64x64 tile, so every tile reads the
// same stream: the low bits of its first 8192 draws (enough for a tile's at most 64 x 64 cells of two draws), draw k at
// bit k % 32 of word k / 32. k_skip_mask builds the mask from them on the device.
void host_skip_stream_bits(uint32_t out[256]);
// The plane-index boundaries of RangeFromPrevious (DenseStereoSgm.cs:94-96); returns whether they are non-decreasing.
bool host_range_bounds(const std::vector<float>& planes, std::vector<float>& b);

// The rsqrtss tables for exponents 127 and 128 (uploaded with the rcp table).
const uint32_t* host_rsqrt_table(bool e128);
// StereoImage.LanczosTable (Lux.Engine/Pipeline/Registration/StereoImage.cs:212-237): 64 phases x 6 taps.
void host_lanczos_table(float out[384]);
// StereoImage.YuvMatrix (StereoImage.cs:140-160): the rows (v, u', t') of ConvertToYUV for a sensor type and neutral.
void host_yuv_matrix(int sensor_type, const float neutral[3], float out[12]);
// Mat4D.Mul (ViewTransform.cs:88-94): row-major double 4x4 product.
void host_mat4_mul(const double* a, const double* b, double* o);

// StereoColorTransfer (color_transfer.cpp): the statistics of one YUVA image, the crop rect and the 4x4 transfer.
struct ColourStats {
  float mean[4], D[4], O[4], N;
};
// CropRect (StereoColorTransfer.cs:32-51) of the rw x rh reference rect, unclamped {x0, y0, x1, y1}.
void host_crop_rect(const lux_calib& ref_view, const lux_calib& view, int rw, int rh, int out[4]);
// Accumulate (:56-75) over w x h pixels of rows `stride` pixels apart, starting at pixel `offset`.
ColourStats host_colour_stats(const float* yuva, int w, int h, int stride, size_t offset);
// Solve (:94-108): the row-major float transfer (the identity below 100 gated pixels in either image).
void host_colour_solve(const ColourStats& work, const ColourStats& ref, float F[16]);

}  // namespace lux
