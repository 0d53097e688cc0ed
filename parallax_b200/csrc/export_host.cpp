// export_host.cpp -- the file formats' host halves: the PLY header, the .spz
// header and gzip wrapper, and the device-to-host copy of the packed body.
//
// The bytes are the reference's writers' (GaussianCloud.cpp:259-306, 414-443,
// 493-550): the same header text, field order and widths, and for .spz the
// same deflate settings (default level, gzip wrapper, window 15, memory level
// 8, default strategy) through the same zlib, so equal planes give equal files.
#include <zlib.h>

#include <cstring>
#include <string>

#include "runtime.h"

namespace pxs {
namespace {

int sh_rest_for_degree(int degree) { return (degree + 1) * (degree + 1) - 1; }

void append_u32(std::vector<uint8_t>* out, uint32_t v) {
  for (int i = 0; i < 4; ++i) out->push_back(static_cast<uint8_t>((v >> (8 * i)) & 0xFF));
}

std::vector<uint8_t> gzip(const std::vector<uint8_t>& in) {
  z_stream stream{};
  if (deflateInit2(&stream, Z_DEFAULT_COMPRESSION, Z_DEFLATED, MAX_WBITS + 16, 8,
                   Z_DEFAULT_STRATEGY) != Z_OK)
    throw Error(PXS_ERR_NO_MEMORY, "deflateInit2 failed");
  std::vector<uint8_t> out(deflateBound(&stream, static_cast<uLong>(in.size())) + 64);
  stream.next_in = const_cast<Bytef*>(in.data());
  stream.avail_in = static_cast<uInt>(in.size());
  stream.next_out = out.data();
  stream.avail_out = static_cast<uInt>(out.size());
  const int rc = deflate(&stream, Z_FINISH);
  const size_t written = out.size() - stream.avail_out;
  deflateEnd(&stream);
  if (rc != Z_STREAM_END) throw Error(PXS_ERR_CUDA, "deflate did not finish");
  out.resize(written);
  return out;
}

}  // namespace

std::vector<uint8_t> export_cloud_bytes(const float* d_params, int n, int S, int sh_degree,
                                        int format, int fractional_bits,
                                        DeviceArray<uint8_t>& body, DeviceArray<int32_t>& fields,
                                        cudaStream_t stream) {
  if (n <= 0) throw Error(PXS_ERR_INVALID, "the cloud is empty");
  if (sh_degree < 0) throw Error(PXS_ERR_INVALID, "negative SH degree");
  std::vector<uint8_t> bytes;
  if (format == PXS_FORMAT_PLY) {
    const int rest_total = sh_rest_for_degree(sh_degree) * 3;
    // plain string building (no iostreams: the library may live in a process
    // whose C++ runtime it does not own)
    std::string text = "ply\nformat binary_little_endian 1.0\n";
    text += "comment generated by Parallax\n";
    text += "element vertex " + std::to_string(n) + "\n";
    text += "property float x\nproperty float y\nproperty float z\n";
    text += "property float nx\nproperty float ny\nproperty float nz\n";
    for (int i = 0; i < 3; ++i) text += "property float f_dc_" + std::to_string(i) + "\n";
    for (int i = 0; i < rest_total; ++i)
      text += "property float f_rest_" + std::to_string(i) + "\n";
    text += "property float opacity\n";
    for (int i = 0; i < 3; ++i) text += "property float scale_" + std::to_string(i) + "\n";
    for (int i = 0; i < 4; ++i) text += "property float rot_" + std::to_string(i) + "\n";
    text += "end_header\n";
    // where each record field comes from (-1: zero)
    std::vector<int32_t> src = {PXS_C_POSITION, PXS_C_POSITION + 1, PXS_C_POSITION + 2,
                                -1, -1, -1, PXS_C_DC, PXS_C_DC + 1, PXS_C_DC + 2};
    for (int i = 0; i < rest_total; ++i) src.push_back(i < 3 * S ? PXS_C_SH_REST + i : -1);
    src.push_back(PXS_C_OPACITY);
    for (int a = 0; a < 3; ++a) src.push_back(PXS_C_LOG_SCALE + a);
    for (int a = 0; a < 4; ++a) src.push_back(PXS_C_ROTATION + a);  // w x y z
    const int nf = static_cast<int>(src.size());
    int32_t* d_src = fields.reserve(src.size());
    PXS_CUDA(cudaMemcpyAsync(d_src, src.data(), src.size() * sizeof(int32_t),
                             cudaMemcpyHostToDevice, stream));
    const size_t body_bytes = static_cast<size_t>(n) * nf * sizeof(float);
    uint8_t* d_body = body.reserve(body_bytes);
    launch_pack_ply(d_params, n, d_src, nf, reinterpret_cast<float*>(d_body), stream);
    PXS_CUDA(cudaGetLastError());
    bytes.resize(text.size() + body_bytes);
    std::memcpy(bytes.data(), text.data(), text.size());
    PXS_CUDA(cudaMemcpyAsync(bytes.data() + text.size(), d_body, body_bytes,
                             cudaMemcpyDeviceToHost, stream));
    PXS_CUDA(cudaStreamSynchronize(stream));
  } else if (format == PXS_FORMAT_SPLAT) {
    const size_t body_bytes = static_cast<size_t>(n) * 32;
    uint8_t* d_body = body.reserve(body_bytes);
    launch_pack_splat(d_params, n, d_body, stream);
    PXS_CUDA(cudaGetLastError());
    bytes.resize(body_bytes);
    PXS_CUDA(cudaMemcpyAsync(bytes.data(), d_body, body_bytes, cudaMemcpyDeviceToHost, stream));
    PXS_CUDA(cudaStreamSynchronize(stream));
  } else if (format == PXS_FORMAT_SPZ) {
    if (sh_degree > 3) throw Error(PXS_ERR_INVALID, ".spz holds SH degrees 0 to 3");
    fractional_bits = std::max(0, std::min(20, fractional_bits));
    const int rest = sh_rest_for_degree(sh_degree);
    const size_t planes = static_cast<size_t>(n) * (9 + 3 + 3 + 1 + 3 + 3 * rest);
    uint8_t* d_body = body.reserve(planes);
    launch_pack_spz(d_params, n, fractional_bits, S, rest, d_body, stream);
    PXS_CUDA(cudaGetLastError());
    std::vector<uint8_t> raw;
    raw.reserve(16 + planes);
    append_u32(&raw, 0x5053474eu);  // "NGSP"
    append_u32(&raw, 2u);           // version
    append_u32(&raw, static_cast<uint32_t>(n));
    raw.push_back(static_cast<uint8_t>(sh_degree));
    raw.push_back(static_cast<uint8_t>(fractional_bits));
    raw.push_back(0);  // not antialiased
    raw.push_back(0);  // reserved
    raw.resize(16 + planes);
    PXS_CUDA(cudaMemcpyAsync(raw.data() + 16, d_body, planes, cudaMemcpyDeviceToHost, stream));
    PXS_CUDA(cudaStreamSynchronize(stream));
    bytes = gzip(raw);
  } else {
    throw Error(PXS_ERR_INVALID, "unknown format");
  }
  return bytes;
}

}  // namespace pxs
