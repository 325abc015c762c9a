// Dump and golden-file formats of the dense stage (Lux.Engine/Pipeline/Registration/StereoAsyncApi.cs:188-262): the
// per-layer files a capture's dense solve writes under a dump prefix (the reference's LUX_DENSE_DUMP), the float image
// format the upsample's override reads back (LUX_DENSE_OVERRIDE, Lux.Engine/Session/ExportBuild.cs:89-96), and the cost
// volume in the reference's memory layout. Host code over the public C ABI: layer fields are read back with
// lux_layer_read, the filtered images are made with lux_sgm_box_filter3, and nothing here changes a result.
//
// Every file starts (where the reference's does) with int32 {w, h, stride, bytes per pixel}, little-endian, stride = w.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/lux_sgm.h"

namespace {

struct File {
  FILE* f = nullptr;
  explicit File(const std::string& path) : f(std::fopen(path.c_str(), "wb")) {}
  ~File() {
    if (f) std::fclose(f);
  }
  bool put(const void* p, size_t n) { return f && (n == 0 || std::fwrite(p, 1, n, f) == n); }
  bool header(int32_t w, int32_t h, int32_t bpp) {
    const int32_t hd[4] = {w, h, w, bpp};
    return put(hd, sizeof hd);
  }
  bool close() {
    const bool ok = f && std::fclose(f) == 0;
    f = nullptr;
    return ok;
  }
};

int write_f32(const std::string& path, const float* data, int32_t w, int32_t h) {
  File f(path);
  if (!f.header(w, h, 4) || !f.put(data, (size_t)w * h * 4) || !f.close()) return LUX_ERR_IO;
  return LUX_OK;
}

int write_rgba8(const std::string& path, const uint8_t* rows, int32_t w, int32_t h, int32_t stride_px) {
  File f(path);
  if (!f.header(w, h, 4)) return LUX_ERR_IO;
  for (int y = 0; y < h; y++)
    if (!f.put(rows + (size_t)y * stride_px * 4, (size_t)w * 4)) return LUX_ERR_IO;
  return f.close() ? LUX_OK : LUX_ERR_IO;
}

template <class T>
int read_field(const lux_layer* L, int32_t field, std::vector<T>& v, size_t n) {
  v.resize(n);
  return n == 0 ? LUX_OK : lux_layer_read(L, field, v.data(), (uint64_t)n * sizeof(T));
}

// A host copy of an image given on the host or the device.
int host_rgba8(const lux_img_rgba8& im, std::vector<uint8_t>& buf, const uint8_t** rows, int32_t* stride_px) {
  if (!im.on_device) {
    *rows = im.data;
    *stride_px = im.stride;
    return LUX_OK;
  }
  buf.resize((size_t)im.w * im.h * 4);
  if (cudaMemcpy2D(buf.data(), (size_t)im.w * 4, im.data, (size_t)im.stride * 4, (size_t)im.w * 4, im.h, cudaMemcpyDeviceToHost) !=
      cudaSuccess)
    return LUX_ERR_CUDA;
  *rows = buf.data();
  *stride_px = im.w;
  return LUX_OK;
}

}  // namespace

extern "C" {

int lux_dump_f32(const char* path, const float* data, int32_t w, int32_t h) {
  if (!path || (!data && (size_t)w * h > 0) || w < 0 || h < 0) return LUX_ERR_ARG;
  return write_f32(path, data, w, h);
}

int lux_load_f32(const char* path, float* out, uint64_t cap_floats, int32_t* w, int32_t* h) {
  if (!path || !w || !h) return LUX_ERR_ARG;
  FILE* f = std::fopen(path, "rb");
  if (!f) return LUX_ERR_IO;
  int32_t hd[4];
  int rc = LUX_OK;
  if (std::fread(hd, 1, sizeof hd, f) != sizeof hd) rc = LUX_ERR_IO;
  else if (hd[3] != 4) rc = LUX_ERR_FORMAT;  // "expected a 4-byte float dump" (StereoAsyncApi.cs:258)
  else if (hd[0] < 0 || hd[1] < 0) rc = LUX_ERR_FORMAT;
  if (rc == LUX_OK) {
    *w = hd[0];
    *h = hd[1];
    const size_t n = (size_t)hd[0] * hd[1];
    if (out) {
      if (n > cap_floats) rc = LUX_ERR_ARG;
      else if (std::fread(out, 4, n, f) != n) rc = LUX_ERR_IO;
    }
  }
  std::fclose(f);
  return rc;
}

int lux_dump_rgba8(const char* path, const lux_img_rgba8* img) {
  if (!path || !img || !img->data || img->w < 0 || img->h < 0 || img->stride < img->w) return LUX_ERR_ARG;
  std::vector<uint8_t> buf;
  const uint8_t* rows = nullptr;
  int32_t stride = 0;
  const int rc = host_rgba8(*img, buf, &rows, &stride);
  return rc ? rc : write_rgba8(path, rows, img->w, img->h, stride);
}

// DumpCostVolume (StereoAsyncApi.cs:227-250): <prefix>_offsets.u32 (header + u32 per pixel, the running byte offset with
// 8 + cap·3 bytes for a computed pixel and 8 + cap·2 for a skipped one, kept to 32 bits as the reference's uint),
// <prefix>_costvol.bin (per pixel {start, count, 1, cap} as u16, cap u16 aggregates, then for computed pixels cap u8
// raw costs) and <prefix>_costvol_pass1.bin with the pass-1 aggregates when the layer kept them.
int lux_dump_cost_volume(const lux_layer* L, const char* prefix) {
  if (!L || !prefix) return LUX_ERR_ARG;
  lux_layer_info in{};
  int rc = lux_layer_get_info(L, &in);
  if (rc) return rc;
  const size_t npx = (size_t)in.w * in.h;
  std::vector<uint16_t> start, count, cap, agg, agg1;
  std::vector<uint8_t> skip, raw;
  std::vector<uint64_t> off;
  if ((rc = read_field(L, LUX_FIELD_START, start, npx)) || (rc = read_field(L, LUX_FIELD_COUNT, count, npx)) ||
      (rc = read_field(L, LUX_FIELD_CAP, cap, npx)) || (rc = read_field(L, LUX_FIELD_SKIP, skip, npx)) ||
      (rc = read_field(L, LUX_FIELD_OFFSETS, off, npx + 1)) || (rc = read_field(L, LUX_FIELD_RAW, raw, in.volume)) ||
      (rc = read_field(L, LUX_FIELD_AGG, agg, in.volume)))
    return rc;  // LUX_FIELD_AGG needs LUX_LAYER_KEEP_AGG on the fast aggregation kernels
  const bool pass1 = read_field(L, LUX_FIELD_AGG_PASS1, agg1, in.volume) == LUX_OK;
  std::vector<uint32_t> boff(npx);
  uint64_t total = 0;
  for (size_t i = 0; i < npx; i++) {
    boff[i] = (uint32_t)total;
    total += 8 + (uint64_t)cap[i] * (skip[i] == 0 ? 3 : 2);
  }
  {
    File f(std::string(prefix) + "_offsets.u32");
    if (!f.header(in.w, in.h, 4) || !f.put(boff.data(), npx * 4) || !f.close()) return LUX_ERR_IO;
  }
  auto write = [&](const std::string& path, const std::vector<uint16_t>& a) {
    File f(path);
    for (size_t i = 0; i < npx; i++) {
      const uint16_t hd[4] = {start[i], count[i], 1, cap[i]};
      if (!f.put(hd, 8) || !f.put(a.data() + off[i], (size_t)cap[i] * 2)) return LUX_ERR_IO;
      if (skip[i] == 0 && !f.put(raw.data() + off[i], cap[i])) return LUX_ERR_IO;
    }
    return f.close() ? LUX_OK : LUX_ERR_IO;
  };
  if ((rc = write(std::string(prefix) + "_costvol.bin", agg))) return rc;
  if (pass1 && (rc = write(std::string(prefix) + "_costvol_pass1.bin", agg1))) return rc;
  return LUX_OK;
}

// The dense dump of StereoAsyncApi.State4And5 (:197-214) for a solved pyramid: per layer <prefix>_dense_L<i>_depth.f32,
// _planes.f32 (raw floats), _skip.u8 (header bpp 1 + w·h bytes); the layer-0 CalibData vector <prefix>_dense_calibs.bin
// (0xa8 bytes per camera: K at 0x00, t at 0x24, R at 0x30, the rest zero); <prefix>_dense_img<k>.img (the inputs) and
// _dense_filt<k>.img (BoxFilter3 of them); <prefix>_dense_L0_guidance.img; the cost volumes of layers 0..cv_max.
int lux_dump_dense(lux_sgm_ctx* ctx, lux_layer* const* layers, int32_t n_layers, int32_t n_cams, const lux_img_rgba8* images,
                   const lux_calib* calibs, const char* prefix, int32_t cv_max) {
  if (!ctx || !layers || n_layers < 1 || n_cams < 1 || !images || !calibs || !prefix) return LUX_ERR_ARG;
  const std::string p(prefix);
  int rc = LUX_OK;
  for (int i = 0; i < n_layers; i++) {
    lux_layer_info in{};
    if ((rc = lux_layer_get_info(layers[i], &in))) return rc;
    const size_t npx = (size_t)in.w * in.h;
    std::vector<float> depth, planes;
    std::vector<uint8_t> skip;
    if ((rc = read_field(layers[i], LUX_FIELD_DEPTH, depth, npx)) || (rc = read_field(layers[i], LUX_FIELD_PLANES, planes, in.n_planes)) ||
        (rc = read_field(layers[i], LUX_FIELD_SKIP, skip, npx)))
      return rc;
    const std::string li = p + "_dense_L" + std::to_string(i);
    if ((rc = write_f32(li + "_depth.f32", depth.data(), in.w, in.h))) return rc;
    {
      File f(li + "_planes.f32");
      if (!f.put(planes.data(), planes.size() * 4) || !f.close()) return LUX_ERR_IO;
    }
    {
      File f(li + "_skip.u8");
      if (!f.header(in.w, in.h, 1) || !f.put(skip.data(), npx) || !f.close()) return LUX_ERR_IO;
    }
    if (i == 0) {
      std::vector<uint8_t> g;
      if ((rc = read_field(layers[i], LUX_FIELD_GUIDANCE, g, npx * 4))) return rc;
      if ((rc = write_rgba8(li + "_guidance.img", g.data(), in.w, in.h, in.w))) return rc;
    }
    if (i <= cv_max && (rc = lux_dump_cost_volume(layers[i], li.c_str()))) return rc;
  }
  {
    std::vector<uint8_t> cb((size_t)n_cams * 0xa8, 0);
    for (int c = 0; c < n_cams; c++) {
      std::memcpy(cb.data() + c * 0xa8, calibs[c].K, 36);
      std::memcpy(cb.data() + c * 0xa8 + 0x24, calibs[c].T, 12);
      std::memcpy(cb.data() + c * 0xa8 + 0x30, calibs[c].R, 36);
    }
    File f(p + "_dense_calibs.bin");
    if (!f.put(cb.data(), cb.size()) || !f.close()) return LUX_ERR_IO;
  }
  for (int k = 0; k < n_cams; k++) {
    const std::string ik = p + "_dense_img" + std::to_string(k) + ".img";
    if ((rc = lux_dump_rgba8(ik.c_str(), &images[k]))) return rc;
    std::vector<uint8_t> filt((size_t)images[k].w * images[k].h * 4);
    if ((rc = lux_sgm_box_filter3(ctx, &images[k], filt.data()))) return rc;
    if ((rc = write_rgba8(p + "_dense_filt" + std::to_string(k) + ".img", filt.data(), images[k].w, images[k].h, images[k].w))) return rc;
  }
  return LUX_OK;
}

}  // extern "C"
