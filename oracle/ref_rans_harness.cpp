// Test-infrastructure only: a C-ABI harness around the reference's own rANS coder
// (MLCodec_extensions_cpp, src/cpp/py_rans/{rans,py_rans}.cpp), compiled from the reference
// sources by oracle/Makefile into oracle/_ref/librans_ref.so.  It is the checker that pins
// the oracle restatement (oracle/rans_oracle.c) and the product coder; nothing in the product
// links it.  Load it with ctypes.PyDLL (the reference returns numpy arrays, so the GIL must be
// held).
//
// The call sequence follows the reference's HT-S worker:
//   encode: reset, set_entropy_coder_parallel, encode_y, encode_z, flush, get_encoded_stream
//           (src/layers/extensions/inference/dmc_hts_proxy.cpp:778-793)
//   decode: set_entropy_coder_parallel, set_stream, decode_z, get_decoded_tensor_cpp,
//           decode_y, get_decoded_tensor_cpp (dmc_hts_proxy.cpp:794-823)
// and the intra worker: encode_y once per mask step (steps 3, 2, 1, 0), then encode_z
// (dmci_proxy.cpp:818-846); decode_z, then one decode_y per step in step order
// (dmci_proxy.cpp:846-870).
#include "py_rans.h"

#include <cstring>
#include <memory>
#include <vector>

namespace {

template <typename T>
std::shared_ptr<std::vector<T>> to_vec(const T* p, int n)
{
    auto v = std::make_shared<std::vector<T>>(n);
    if (n > 0) {
        std::memcpy(v->data(), p, sizeof(T) * n);
    }
    return v;
}

}  // namespace

extern "C" {

// Returns the number of cdf entries written (n + 1).
int ref_pmf_to_quantized_cdf(const float* pmf, int n, uint32_t* cdf_out)
{
    std::vector<float> p(pmf, pmf + n);
    auto cdf = pmf_to_quantized_cdf(p);
    std::memcpy(cdf_out, cdf.data(), cdf.size() * sizeof(uint32_t));
    return static_cast<int>(cdf.size());
}

// cdf tables are [n_cdf, stride] int32 with lengths [n_cdf]; index 0 = z (bit estimator),
// index 1 = y (gaussian).  Returns the number of bytes written to out, or -1 if out_cap is
// too small.
int ref_encode(const int32_t* cdf_z, const int32_t* len_z, int n_z_cdf, int z_stride,
               const int32_t* cdf_y, const int32_t* len_y, int n_y_cdf, int y_stride,
               const int16_t* y_sym, int n_y, const int8_t* z_sym, int n_z, int z_cdf_offset,
               int z_ch, int ec_parallel, uint8_t* out, int out_cap)
{
    RansEncoder enc;
    enc.set_cdf(to_vec(cdf_z, n_z_cdf * z_stride), to_vec(len_z, n_z_cdf), 0);
    enc.set_cdf(to_vec(cdf_y, n_y_cdf * y_stride), to_vec(len_y, n_y_cdf), 1);
    enc.reset();
    enc.set_entropy_coder_parallel(ec_parallel);
    enc.encode_y(to_vec(y_sym, n_y), n_y);
    enc.encode_z(to_vec(z_sym, n_z), z_cdf_offset, z_ch);
    enc.flush();
    py::array_t<uint8_t> s = enc.get_encoded_stream();
    const int n = static_cast<int>(s.size());
    if (n > out_cap) {
        return -1;
    }
    std::memcpy(out, s.data(), n);
    return n;
}

int ref_decode(const int32_t* cdf_z, const int32_t* len_z, int n_z_cdf, int z_stride,
               const int32_t* cdf_y, const int32_t* len_y, int n_y_cdf, int y_stride,
               const uint8_t* stream, int stream_size, const uint8_t* y_idx, int n_y, int n_z,
               int z_cdf_offset, int z_ch, int ec_parallel, int8_t* y_out, int8_t* z_out)
{
    RansDecoder dec;
    dec.set_cdf(to_vec(cdf_z, n_z_cdf * z_stride), to_vec(len_z, n_z_cdf), 0);
    dec.set_cdf(to_vec(cdf_y, n_y_cdf * y_stride), to_vec(len_y, n_y_cdf), 1);
    dec.set_entropy_coder_parallel(ec_parallel);
    dec.set_stream(stream, stream_size);
    dec.decode_z(n_z, z_cdf_offset, z_ch);
    auto z = dec.get_decoded_tensor_cpp();
    std::memcpy(z_out, z->data(), n_z);
    dec.decode_y(to_vec(y_idx, n_y), n_y);
    auto y = dec.get_decoded_tensor_cpp();
    std::memcpy(y_out, y->data(), n_y);
    return 0;
}

// Several y segments (lengths y_counts, concatenated in y_sym in coding order), then z.
int ref_encode_segments(const int32_t* cdf_z, const int32_t* len_z, int n_z_cdf, int z_stride,
                        const int32_t* cdf_y, const int32_t* len_y, int n_y_cdf, int y_stride,
                        const int16_t* y_sym, const int* y_counts, int n_seg, const int8_t* z_sym,
                        int n_z, int z_cdf_offset, int z_ch, int ec_parallel, uint8_t* out,
                        int out_cap)
{
    RansEncoder enc;
    enc.set_cdf(to_vec(cdf_z, n_z_cdf * z_stride), to_vec(len_z, n_z_cdf), 0);
    enc.set_cdf(to_vec(cdf_y, n_y_cdf * y_stride), to_vec(len_y, n_y_cdf), 1);
    enc.reset();
    enc.set_entropy_coder_parallel(ec_parallel);
    for (int g = 0; g < n_seg; ++g) {
        enc.encode_y(to_vec(y_sym, y_counts[g]), y_counts[g]);
        y_sym += y_counts[g];
    }
    enc.encode_z(to_vec(z_sym, n_z), z_cdf_offset, z_ch);
    enc.flush();
    py::array_t<uint8_t> s = enc.get_encoded_stream();
    const int n = static_cast<int>(s.size());
    if (n > out_cap) {
        return -1;
    }
    std::memcpy(out, s.data(), n);
    return n;
}

// Incremental decoding: open, decode_z, decode_y (any number of times), close.
void* ref_dec_open(const int32_t* cdf_z, const int32_t* len_z, int n_z_cdf, int z_stride,
                   const int32_t* cdf_y, const int32_t* len_y, int n_y_cdf, int y_stride,
                   const uint8_t* stream, int stream_size, int ec_parallel)
{
    auto* dec = new RansDecoder();
    dec->set_cdf(to_vec(cdf_z, n_z_cdf * z_stride), to_vec(len_z, n_z_cdf), 0);
    dec->set_cdf(to_vec(cdf_y, n_y_cdf * y_stride), to_vec(len_y, n_y_cdf), 1);
    dec->set_entropy_coder_parallel(ec_parallel);
    dec->set_stream(stream, stream_size);
    return dec;
}

int ref_dec_z(void* h, int n_z, int z_cdf_offset, int z_ch, int8_t* z_out)
{
    auto* dec = static_cast<RansDecoder*>(h);
    dec->decode_z(n_z, z_cdf_offset, z_ch);
    auto z = dec->get_decoded_tensor_cpp();
    std::memcpy(z_out, z->data(), n_z);
    return 0;
}

int ref_dec_y(void* h, const uint8_t* y_idx, int n_y, int8_t* y_out)
{
    auto* dec = static_cast<RansDecoder*>(h);
    dec->decode_y(to_vec(y_idx, n_y), n_y);
    auto y = dec->get_decoded_tensor_cpp();
    if (n_y > 0) {
        std::memcpy(y_out, y->data(), n_y);
    }
    return 0;
}

void ref_dec_close(void* h) { delete static_cast<RansDecoder*>(h); }

}  // extern "C"
