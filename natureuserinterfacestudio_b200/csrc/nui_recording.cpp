// Recorded frames: the reference's frame file format (NuiFileIOUtilities.cpp:13-161) and
// its recording layout (NuiFrameLoader.cpp:26-92), so that recorded sessions can feed the
// tracking and serving paths.
//
// A frame image file holds  int64 timestamp, uint32 width, uint32 height, uint32 stored
// size, payload;  the payload is the raw pixels (width * height * pixel bytes) or, when the
// stored size differs from that, their zlib stream (compress2 at Z_BEST_SPEED when written).
// A camera file holds four floats fx, fy, cx, cy.  A recording is a directory of
// <n>.depth (uint16 millimetres), <n>.color (BGRA) and <n>.camIntri files, n = 0, 1, ...
#include <zlib.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/nui_b200.h"

namespace {
struct File {
  FILE* f;
  explicit File(const char* path, const char* mode) : f(std::fopen(path, mode)) {}
  ~File() {
    if (f) std::fclose(f);
  }
};
}  // namespace

extern "C" {

NUI_API nui_status nui_frame_file_write(const char* path, int compressed, int64_t timestamp, uint32_t width,
                                        uint32_t height, const void* pixels, uint32_t pixel_bytes) {
  if (!path || !pixels || width == 0 || height == 0 || pixel_bytes == 0) return NUI_ERR_INVALID_ARG;
  const uint64_t raw64 = (uint64_t)width * height * pixel_bytes;
  if (raw64 > 0xffffffffull) return NUI_ERR_INVALID_ARG;
  const uint32_t raw = (uint32_t)raw64;
  File out(path, "wb");
  if (!out.f) return NUI_ERR_INVALID_ARG;
  bool ok = std::fwrite(&timestamp, 8, 1, out.f) == 1 && std::fwrite(&width, 4, 1, out.f) == 1 &&
            std::fwrite(&height, 4, 1, out.f) == 1;
  std::vector<Bytef> z;
  uLongf zsize = 0;
  bool use_z = false;
  if (compressed) {
    zsize = compressBound(raw);
    z.resize(zsize);
    use_z = compress2(z.data(), &zsize, (const Bytef*)pixels, raw, Z_BEST_SPEED) == Z_OK;
  }
  if (use_z) {
    const uint32_t stored = (uint32_t)zsize;
    ok = ok && std::fwrite(&stored, 4, 1, out.f) == 1 && std::fwrite(z.data(), 1, zsize, out.f) == zsize;
  } else {
    ok = ok && std::fwrite(&raw, 4, 1, out.f) == 1 && std::fwrite(pixels, 1, raw, out.f) == raw;
  }
  return ok ? NUI_OK : NUI_ERR_DEVICE;
}

NUI_API nui_status nui_frame_file_header(const char* path, int64_t* timestamp, uint32_t* width, uint32_t* height) {
  if (!path) return NUI_ERR_INVALID_ARG;
  File in(path, "rb");
  if (!in.f) return NUI_ERR_INVALID_ARG;
  int64_t ts = 0;
  uint32_t w = 0, h = 0;
  if (std::fread(&ts, 8, 1, in.f) != 1 || std::fread(&w, 4, 1, in.f) != 1 || std::fread(&h, 4, 1, in.f) != 1)
    return NUI_ERR_INVALID_ARG;
  if (timestamp) *timestamp = ts;
  if (width) *width = w;
  if (height) *height = h;
  return NUI_OK;
}

NUI_API nui_status nui_frame_file_read(const char* path, void* pixels, uint32_t bytes) {
  if (!path || !pixels || bytes == 0) return NUI_ERR_INVALID_ARG;
  File in(path, "rb");
  if (!in.f) return NUI_ERR_INVALID_ARG;
  uint32_t stored = 0;
  if (std::fseek(in.f, 16, SEEK_SET) != 0 || std::fread(&stored, 4, 1, in.f) != 1) return NUI_ERR_INVALID_ARG;
  if (stored == bytes) return std::fread(pixels, 1, bytes, in.f) == bytes ? NUI_OK : NUI_ERR_INVALID_ARG;
  std::vector<Bytef> z(stored);
  if (std::fread(z.data(), 1, stored, in.f) != stored) return NUI_ERR_INVALID_ARG;
  uLongf out = bytes;
  if (uncompress((Bytef*)pixels, &out, z.data(), stored) != Z_OK || out != bytes) return NUI_ERR_INVALID_ARG;
  return NUI_OK;
}

NUI_API nui_status nui_camera_file_write(const char* path, const float* fx_fy_cx_cy) {
  if (!path || !fx_fy_cx_cy) return NUI_ERR_INVALID_ARG;
  File out(path, "wb");
  if (!out.f) return NUI_ERR_INVALID_ARG;
  return std::fwrite(fx_fy_cx_cy, 4, 4, out.f) == 4 ? NUI_OK : NUI_ERR_DEVICE;
}

NUI_API nui_status nui_camera_file_read(const char* path, float* fx_fy_cx_cy) {
  if (!path || !fx_fy_cx_cy) return NUI_ERR_INVALID_ARG;
  File in(path, "rb");
  if (!in.f) return NUI_ERR_INVALID_ARG;
  return std::fread(fx_fy_cx_cy, 4, 4, in.f) == 4 ? NUI_OK : NUI_ERR_INVALID_ARG;
}

NUI_API nui_status nui_recording_frame(const char* dir, int index, uint16_t* depth_mm, uint8_t* bgra,
                                       float* fx_fy_cx_cy, int64_t* timestamp, uint32_t width, uint32_t height) {
  if (!dir || index < 0) return NUI_ERR_INVALID_ARG;
  const std::string base = std::string(dir) + "/" + std::to_string(index);
  bool any = false;
  if (depth_mm) {
    uint32_t w = 0, h = 0;
    if (nui_frame_file_header((base + ".depth").c_str(), timestamp, &w, &h) == NUI_OK) {
      if (w != width || h != height) return NUI_ERR_INVALID_ARG;
      if (nui_frame_file_read((base + ".depth").c_str(), depth_mm, width * height * 2) != NUI_OK)
        return NUI_ERR_INVALID_ARG;
      any = true;
    }
  }
  if (bgra) {
    uint32_t w = 0, h = 0;
    if (nui_frame_file_header((base + ".color").c_str(), depth_mm ? nullptr : timestamp, &w, &h) == NUI_OK) {
      if (w != width || h != height) return NUI_ERR_INVALID_ARG;
      if (nui_frame_file_read((base + ".color").c_str(), bgra, width * height * 4) != NUI_OK)
        return NUI_ERR_INVALID_ARG;
      any = true;
    }
  }
  if (fx_fy_cx_cy && nui_camera_file_read((base + ".camIntri").c_str(), fx_fy_cx_cy) == NUI_OK) any = true;
  return any ? NUI_OK : NUI_ERR_INVALID_ARG;  // no file of that frame: the end of the recording
}

}  // extern "C"
