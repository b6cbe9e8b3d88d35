// MLCodec-compatible rANS coder (host C++), byte-identical to the reference's
// MLCodec_extensions_cpp (src/cpp/py_rans/rans.cpp, py_rans.cpp).
//
// Format: 32-bit state, 16-bit probabilities, L = 2^23, byte-wise renormalisation, a 2-bit
// bypass escape for |v| >= max_value; y symbols use table index (sym & 0xff) of the Gaussian
// tables, z symbols table (i % ch) + cdf_offset of the bit-estimator tables.  Up to 8
// sub-streams: symbol ranges split evenly, sub-stream pairs merged as forward + reversed with
// shared trailing bytes overlapped, and an int32 offset header (py_rans.cpp:156-249).
#pragma once

#include <stdint.h>

#include <string>
#include <vector>

namespace dcvc {

constexpr int kMaxEcParallel = 8;
constexpr int kMinSymbolsPerStream = 32768;

// ec_parallel for a symbol count (dmc_common.cpp:31-35).
int ec_parallel_for(int symbol_count);

// pmf -> quantised CDF with 16-bit precision (py_rans.cpp:35-94).  Returns n+1 entries or an
// empty vector if the pmf cannot be made valid.
std::vector<uint32_t> pmf_to_quantized_cdf(const float* pmf, int n);

// Encoder form of one symbol: the state update x -> ((x / freq) << 16) + x % freq + start written
// as x + bias + q * cmpl with q = x / freq from a multiply-high by a rounded-up reciprocal and a
// shift (exact for the encoder's x < 2^31; the published method of Giesen's ryg_rans).
struct RansEncSym {
    uint32_t x_max;  // freq << 15: renormalise while x >= x_max (0: zero frequency)
    uint32_t rcp;
    uint32_t bias;
    uint16_t cmpl;   // (1 << 16) - freq
    uint16_t shift;
};

struct RansTable {
    int count = 0;   // number of tables
    int stride = 0;  // int32 entries per table
    std::vector<int32_t> cdf;       // [count * stride]
    std::vector<int32_t> max_value; // cdf_length - 2
    std::vector<uint32_t> enc;      // [count * stride]: start | (freq << 16)
    std::vector<RansEncSym> esym;   // [count * stride]
};

// The two table sets of a coder: index 0 = z (bit estimator), index 1 = y (Gaussian).
class RansTables {
public:
    bool set(int index, const int32_t* cdf, const int32_t* lengths, int count, int stride,
             std::string* err);
    bool ready() const { return t_[0].count > 0 && t_[1].count > 0; }
    const RansTable& z() const { return t_[0]; }
    const RansTable& y() const { return t_[1]; }

private:
    RansTable t_[2];
};

// One encoded payload.  Segments are coded in the order they are added; every segment is split
// evenly over the ec_parallel sub-streams and each sub-stream codes its slices back to front, as
// the reference's per-sub-stream task queues do (rans.cpp:239-294, py_rans.cpp:104-135).
class RansEncoderSession {
public:
    void reset(int ec_parallel);
    // y symbols: (value << 8) + table index, int16.  With copy = false the symbols are borrowed
    // and must stay valid until finish().
    void add_y(const int16_t* sym, int n, bool copy = true);
    // z symbols use table (i % ch) + cdf_offset.
    void add_z(const int8_t* sym, int n, int cdf_offset, int ch, bool copy = true);
    // Codes all segments and merges the sub-streams into the container.  An exception in any
    // sub-stream task (e.g. a failed allocation) is caught: finish returns false with the
    // message and fault() is true.
    bool finish(const RansTables& tables, std::vector<uint8_t>* out, std::string* err);
    int ec_parallel() const { return ecp_; }
    bool fault() const { return fault_; }

private:
    bool finish_tasks(const RansTables& tables, std::vector<uint8_t>* out, std::string* err);
    bool fault_ = false;
    struct Segment {
        bool is_y;
        const int16_t* y;
        const int8_t* z;
        int n;
        int cdf_offset;
        int ch;
        std::vector<int16_t> own_y;
        std::vector<int8_t> own_z;
    };
    int ecp_ = 1;
    std::vector<Segment> segs_;
};

// Incremental decoder over one payload: segments are decoded in the reverse order of encoding.
class RansDecoderSession {
public:
    bool begin(const uint8_t* data, int size, int ec_parallel, std::string* err);
    bool decode_z(const RansTables& tables, int n, int cdf_offset, int ch, int8_t* out,
                  std::string* err);
    bool decode_y(const RansTables& tables, const uint8_t* idx, int n, int8_t* out,
                  std::string* err);
    // true when the last call failed on an exception in the coder (not on the stream's bytes)
    bool fault() const { return fault_; }

private:
    bool begin_tasks(const uint8_t* data, int size, int ec_parallel, std::string* err);
    bool decode_z_tasks(const RansTables& tables, int n, int cdf_offset, int ch, int8_t* out,
                        std::string* err);
    bool decode_y_tasks(const RansTables& tables, const uint8_t* idx, int n, int8_t* out,
                        std::string* err);
    bool fault_ = false;
    struct Reader {
        const uint8_t* p = nullptr;
        const uint8_t* end = nullptr;
        uint32_t x = 0;
        bool overrun = false;
    };
    int ecp_ = 0;
    std::vector<uint8_t> parts_[kMaxEcParallel];
    Reader r_[kMaxEcParallel];
};

// Failure-path testing: the next coder task of sub-stream `sub_stream` (0 .. 7) throws inside
// its worker, as an allocation failure there would; -1 cancels a pending injection.
void rans_inject_task_fault(int sub_stream);

}  // namespace dcvc
