#include "rans_coder.h"

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <exception>
#include <functional>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>

#include <unistd.h>

namespace dcvc {

namespace {

constexpr int kScaleBits = 16;
constexpr uint32_t kRansL = 1u << 23;
constexpr int kRenormShift = 23 - kScaleBits + 8;  // 15
constexpr uint32_t kBypassMax = 3;                 // 2-bit bypass digits
constexpr uint32_t kBypassXMax = (1u << (kScaleBits - 2)) << kRenormShift;

// Sub-stream writer: bytes are produced back to front.  Each coding thread works on a Writer of
// its own stack (moved out when done): writers side by side in one array would share cache lines
// that every symbol updates.
struct Writer {
    std::unique_ptr<uint8_t[]> buf;  // not zero-filled: every byte handed out is written
    size_t cap = 0;
    size_t pos = 0;
    uint32_t x = kRansL;
    bool overflow = false;
    bool zero_freq = false;  // a symbol with zero probability in its table (cannot be coded)

    void init(size_t n)
    {
        buf.reset(new uint8_t[n]);
        cap = n;
        pos = n;
        x = kRansL;
        overflow = false;
        zero_freq = false;
    }
    inline void byte(uint8_t b)
    {
        if (pos == 0) {
            overflow = true;
            return;
        }
        buf[--pos] = b;
    }
    inline void put(const RansEncSym& e)
    {
        if (e.x_max == 0) {
            zero_freq = true;
            return;
        }
        while (x >= e.x_max) {
            byte(static_cast<uint8_t>(x));
            x >>= 8;
        }
        const uint32_t q =
            static_cast<uint32_t>((static_cast<uint64_t>(x) * e.rcp) >> 32) >> e.shift;
        x += e.bias + q * e.cmpl;
    }
    inline void bits(uint32_t v)
    {
        while (x >= kBypassXMax) {
            byte(static_cast<uint8_t>(x));
            x >>= 8;
        }
        x = (x << 2) | v;
    }
    inline void symbol(int32_t s, int32_t maxv, const RansEncSym* enc)
    {
        int32_t v = (s < 0 ? -s : s) * 2 - (s > 0);
        if (v >= maxv) {
            const uint32_t raw = static_cast<uint32_t>(v - maxv);
            uint32_t bins[40];
            int nb = 0;
            int digits = 0;
            while (digits < 16 && (raw >> (digits * 2)) != 0) {
                ++digits;
            }
            int32_t cnt = digits;
            while (cnt >= static_cast<int32_t>(kBypassMax)) {
                bins[nb++] = kBypassMax;
                cnt -= kBypassMax;
            }
            bins[nb++] = static_cast<uint32_t>(cnt);
            for (int j = 0; j < digits; ++j) {
                bins[nb++] = (raw >> (2 * j)) & kBypassMax;
            }
            for (int j = nb - 1; j >= 0; --j) {
                bits(bins[j]);
            }
            v = maxv;
        }
        put(enc[v]);
    }
    void flush()
    {
        for (int k = 3; k >= 0; --k) {
            byte(static_cast<uint8_t>(x >> (8 * k)));
        }
    }
    const uint8_t* data() const { return buf.get() + pos; }
    int size() const { return static_cast<int>(cap - pos); }
};

inline void split(int n, int parts, int i, int* begin, int* end)
{
    const int s = n / parts;
    *begin = s * i;
    *end = (i < parts - 1) ? *begin + s : n;
}

int shared_tail(const uint8_t* a, int na, const uint8_t* b, int nb)
{
    const int lim = std::min({na, nb, 8});
    int k = 0;
    for (int i = 0; i < lim; ++i) {
        if (a[na - 1 - i] != 0 || b[nb - 1 - i] != 0) {
            break;
        }
        ++k;
    }
    if (k == 0 && a[na - 1] == b[nb - 1]) {
        k = 1;
    }
    return k;
}

// Sub-stream index whose next task throws (failure-path tests); -1: none.
std::atomic<int> g_inject_task{-1};

// Runs task i of a coder call, throwing first when a fault is injected for it.
template <typename F>
void run_task(F& f, int i)
{
    int want = i;
    if (g_inject_task.load(std::memory_order_relaxed) == i &&
        g_inject_task.compare_exchange_strong(want, -1)) {
        throw std::runtime_error("injected fault in sub-stream task " + std::to_string(i));
    }
    f(i);
}

// Persistent workers for the sub-stream tasks of one calling thread (a codec stream's host
// thread): spawning threads on every call cost as much as coding a small payload.  Workers are
// created on first use, one per extra sub-stream, and joined when the calling thread exits; a
// forked child gets a pool of its own.
class WorkerPool {
public:
    ~WorkerPool()
    {
        {
            std::lock_guard<std::mutex> lk(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : th_) {
            t.join();
        }
    }
    // Runs f(0) on the calling thread and f(1 .. n-1) on the workers.  Every task runs to the
    // end even when one throws; the first exception is rethrown here after all have finished,
    // so no task outlives the caller's frame and no worker terminates the process.
    void run(int n, const std::function<void(int)>& f)
    {
        while (static_cast<int>(th_.size()) < n - 1) {
            th_.emplace_back([this] { work(); });
        }
        {
            std::lock_guard<std::mutex> lk(m_);
            fn_ = &f;
            next_ = 1;
            n_ = n;
            left_ = n - 1;
            first_error_ = nullptr;
        }
        cv_.notify_all();
        call(f, 0);
        std::unique_lock<std::mutex> lk(m_);
        done_.wait(lk, [this] { return left_ == 0; });
        fn_ = nullptr;
        if (first_error_) {
            std::exception_ptr e = first_error_;
            first_error_ = nullptr;
            lk.unlock();
            std::rethrow_exception(e);
        }
    }

private:
    void work()
    {
        std::unique_lock<std::mutex> lk(m_);
        for (;;) {
            cv_.wait(lk, [this] { return stop_ || next_ < n_; });
            if (stop_) {
                return;
            }
            const int i = next_++;
            const std::function<void(int)>* f = fn_;
            lk.unlock();
            call(*f, i);
            lk.lock();
            if (--left_ == 0) {
                done_.notify_one();
            }
        }
    }

    // one task; an exception is kept (the first of the call) instead of escaping the thread
    void call(const std::function<void(int)>& f, int i)
    {
        try {
            run_task(f, i);
        } catch (...) {
            std::lock_guard<std::mutex> lk(m_);
            if (!first_error_) {
                first_error_ = std::current_exception();
            }
        }
    }

    std::mutex m_;
    std::condition_variable cv_, done_;
    std::vector<std::thread> th_;
    const std::function<void(int)>* fn_ = nullptr;
    int next_ = 0, n_ = 0, left_ = 0;
    bool stop_ = false;
    std::exception_ptr first_error_;
};

template <typename F>
void run_parallel(int n, F&& f)
{
    if (n == 1) {
        run_task(f, 0);
        return;
    }
    thread_local std::unique_ptr<WorkerPool> pool;
    thread_local pid_t owner = 0;
    if (pool == nullptr || owner != getpid()) {
        (void)pool.release();  // a pool inherited through fork() has no threads: leave it
        pool.reset(new WorkerPool());
        owner = getpid();
    }
    const std::function<void(int)> fn = std::forward<F>(f);
    pool->run(n, fn);
}

}  // namespace

int ec_parallel_for(int symbol_count)
{
    int n = symbol_count / kMinSymbolsPerStream;
    return std::max(1, std::min(kMaxEcParallel, n));
}

std::vector<uint32_t> pmf_to_quantized_cdf(const float* pmf, int n)
{
    const uint32_t prob_max = 1u << 16;
    const int m = n + 1;
    std::vector<uint32_t> cdf(m, 0);
    for (int i = 0; i < n; ++i) {
        const float prod = pmf[i] * static_cast<float>(prob_max);
        cdf[i + 1] = static_cast<uint32_t>(static_cast<double>(prod) + 0.5);
    }
    int total = 0;
    for (int i = 0; i < m; ++i) {
        total += static_cast<int>(cdf[i]);
    }
    if (total <= 0) {
        return {};
    }
    for (int i = 0; i < m; ++i) {
        cdf[i] = static_cast<uint32_t>((static_cast<uint64_t>(prob_max) * cdf[i]) /
                                       static_cast<uint32_t>(total));
    }
    for (int i = 1; i < m; ++i) {
        cdf[i] += cdf[i - 1];
    }
    cdf[m - 1] = prob_max;
    for (int i = 0; i < m - 1; ++i) {
        if (cdf[i] + 1 > cdf[i + 1]) {
            uint32_t best_freq = ~0u;
            int best = -1;
            for (int j = 0; j < m - 1; ++j) {
                const uint32_t f = cdf[j + 1] - cdf[j];
                if (f >= 2 && f < best_freq) {
                    best_freq = f;
                    best = j;
                }
            }
            if (best < 0) {
                return {};
            }
            if (best < i) {
                for (int j = best + 1; j <= i; ++j) {
                    cdf[j] -= 1;
                }
            } else {
                for (int j = i + 1; j <= best; ++j) {
                    cdf[j] += 1;
                }
            }
        }
    }
    return cdf;
}

bool RansTables::set(int index, const int32_t* cdf, const int32_t* lengths, int count, int stride,
                     std::string* err)
{
    if (index < 0 || index > 1 || count <= 0 || stride < 3) {
        *err = "rANS tables: bad index, count or stride";
        return false;
    }
    RansTable t;
    t.count = count;
    t.stride = stride;
    t.cdf.assign(cdf, cdf + static_cast<size_t>(count) * stride);
    t.max_value.resize(count);
    t.enc.assign(static_cast<size_t>(count) * stride, 0);
    t.esym.assign(static_cast<size_t>(count) * stride, RansEncSym{});
    for (int i = 0; i < count; ++i) {
        const int len = lengths[i];
        if (len < 3 || len > stride) {
            *err = "rANS tables: cdf length out of range";
            return false;
        }
        t.max_value[i] = static_cast<int8_t>(len - 2);
        const int32_t* c = t.cdf.data() + static_cast<size_t>(i) * stride;
        for (int j = 0; j + 1 < stride; ++j) {
            const uint32_t start = static_cast<uint16_t>(c[j]);
            const uint32_t freq = static_cast<uint16_t>(c[j + 1] - c[j]);
            t.enc[static_cast<size_t>(i) * stride + j] = start | (freq << 16);
            RansEncSym& es = t.esym[static_cast<size_t>(i) * stride + j];
            es.x_max = freq << kRenormShift;
            es.cmpl = static_cast<uint16_t>((1u << kScaleBits) - freq);
            if (freq < 2) {
                // q = x - 1 from the multiply-high, made up for by the bias
                es.rcp = ~0u;
                es.shift = 0;
                es.bias = start + (1u << kScaleBits) - 1;
            } else {
                uint32_t sh = 0;
                while (freq > (1u << sh)) {
                    ++sh;
                }
                es.rcp = static_cast<uint32_t>(((uint64_t{1} << (sh + 31)) + freq - 1) / freq);
                es.shift = static_cast<uint16_t>(sh - 1);
                es.bias = start;
            }
        }
    }
    t_[index] = std::move(t);
    return true;
}

void RansEncoderSession::reset(int ec_parallel)
{
    ecp_ = ec_parallel;
    segs_.clear();
}

void RansEncoderSession::add_y(const int16_t* sym, int n, bool copy)
{
    Segment s{};
    s.is_y = true;
    s.n = n;
    if (copy) {
        s.own_y.assign(sym, sym + n);
        s.y = s.own_y.data();
    } else {
        s.y = sym;
    }
    segs_.push_back(std::move(s));
    if (copy) {
        segs_.back().y = segs_.back().own_y.data();
    }
}

void RansEncoderSession::add_z(const int8_t* sym, int n, int cdf_offset, int ch, bool copy)
{
    Segment s{};
    s.is_y = false;
    s.n = n;
    s.cdf_offset = cdf_offset;
    s.ch = ch;
    if (copy) {
        s.own_z.assign(sym, sym + n);
    } else {
        s.z = sym;
    }
    segs_.push_back(std::move(s));
    if (copy) {
        segs_.back().z = segs_.back().own_z.data();
    }
}

namespace {

// Converts an exception thrown by a coder call into its false / err form.
template <typename F>
bool guarded(bool* fault, std::string* err, F&& body)
{
    *fault = false;
    try {
        return body();
    } catch (const std::bad_alloc&) {
        *err = "rANS: out of host memory";
    } catch (const std::exception& e) {
        *err = std::string("rANS: ") + e.what();
    }
    *fault = true;
    return false;
}

}  // namespace

bool RansEncoderSession::finish(const RansTables& tables, std::vector<uint8_t>* out,
                                std::string* err)
{
    return guarded(&fault_, err, [&] { return finish_tasks(tables, out, err); });
}

bool RansEncoderSession::finish_tasks(const RansTables& tables, std::vector<uint8_t>* out,
                                      std::string* err)
{
    if (!tables.ready()) {
        *err = "rANS encode: tables not set";
        return false;
    }
    const int ecp = ecp_;
    if (ecp < 1 || ecp > kMaxEcParallel) {
        *err = "rANS encode: ec_parallel must be in [1, 8]";
        return false;
    }
    const RansTable& ty = tables.y();
    const RansTable& tz = tables.z();
    size_t cap[kMaxEcParallel] = {0};
    for (const Segment& sg : segs_) {
        if (sg.n < 0 || (!sg.is_y && (sg.ch < 1 || sg.cdf_offset < 0 ||
                                      (sg.n > 0 && sg.cdf_offset + sg.ch > tz.count)))) {
            *err = "rANS encode: bad segment arguments";
            return false;
        }
        for (int i = 0; i < ecp; ++i) {
            int b, e;
            split(sg.n, ecp, i, &b, &e);
            cap[i] += static_cast<size_t>(e - b) * 4;
        }
    }
    Writer w[kMaxEcParallel];
    bool bad_index[kMaxEcParallel] = {false};
    run_parallel(ecp, [&](int i) {
        Writer lw;
        lw.init(cap[i] + 16);
        for (const Segment& sg : segs_) {
            int b, e;
            split(sg.n, ecp, i, &b, &e);
            if (sg.is_y) {
                for (int k = e - 1; k >= b; --k) {
                    const int16_t c = sg.y[k];
                    const int idx = c & 0xff;
                    if (idx >= ty.count) {
                        bad_index[i] = true;
                        return;
                    }
                    const int32_t s = static_cast<int8_t>(c >> 8);
                    lw.symbol(s, ty.max_value[idx],
                              ty.esym.data() + static_cast<size_t>(idx) * ty.stride);
                }
            } else {
                // table (k % ch) + cdf_offset, the channel stepped down with k (no division per
                // symbol)
                int chn = e > b ? (e - 1) % sg.ch : 0;
                for (int k = e - 1; k >= b; --k) {
                    const int t = chn + sg.cdf_offset;
                    lw.symbol(sg.z[k], tz.max_value[t],
                              tz.esym.data() + static_cast<size_t>(t) * tz.stride);
                    chn = chn == 0 ? sg.ch - 1 : chn - 1;
                }
            }
        }
        lw.flush();
        w[i] = std::move(lw);
    });
    for (int i = 0; i < ecp; ++i) {
        if (bad_index[i]) {
            *err = "rANS encode: y symbol names a CDF table out of range";
            return false;
        }
        if (w[i].overflow) {
            *err = "rANS encode: sub-stream buffer overflow";
            return false;
        }
        if (w[i].zero_freq) {
            *err = "rANS encode: a symbol has zero probability in its table";
            return false;
        }
    }
    out->clear();
    if (ecp == 1) {
        out->assign(w[0].data(), w[0].data() + w[0].size());
        return true;
    }
    const int pairs = ecp / 2;
    const bool tail = (ecp % 2) != 0;
    int same[kMaxEcParallel / 2], gsz[kMaxEcParallel / 2];
    for (int p = 0; p < pairs; ++p) {
        const Writer& a = w[2 * p];
        const Writer& b = w[2 * p + 1];
        same[p] = shared_tail(a.data(), a.size(), b.data(), b.size());
        gsz[p] = a.size() + b.size() - same[p];
    }
    const int noff = pairs - 1 + (tail ? 1 : 0);
    size_t total = static_cast<size_t>(noff) * 4;
    for (int p = 0; p < pairs; ++p) {
        total += gsz[p];
    }
    if (tail) {
        total += w[ecp - 1].size();
    }
    out->resize(total);
    uint8_t* o = out->data();
    int32_t cum = gsz[0];
    for (int k = 0; k < noff; ++k) {
        std::memcpy(o + 4 * k, &cum, 4);
        if (k + 1 < pairs) {
            cum += gsz[k + 1];
        }
    }
    size_t pos = static_cast<size_t>(noff) * 4;
    for (int p = 0; p < pairs; ++p) {
        const Writer& a = w[2 * p];
        const Writer& b = w[2 * p + 1];
        std::memcpy(o + pos, a.data(), a.size());
        const int nb = b.size() - same[p];
        std::reverse_copy(b.data(), b.data() + nb, o + pos + a.size());
        pos += gsz[p];
    }
    if (tail) {
        std::memcpy(o + pos, w[ecp - 1].data(), w[ecp - 1].size());
    }
    return true;
}

namespace {

inline uint8_t rd_next(const uint8_t*& p, const uint8_t* end, bool& overrun)
{
    if (p >= end) {
        overrun = true;
        return 0;
    }
    return *p++;
}

inline uint32_t rd_bits(uint32_t& x, const uint8_t*& p, const uint8_t* end, bool& overrun)
{
    const uint32_t v = x & kBypassMax;
    x >>= 2;
    if (x < kRansL) {
        x = (x << 8) | rd_next(p, end, overrun);
    }
    return v;
}

inline int8_t rd_symbol(uint32_t& x, const uint8_t*& p, const uint8_t* end, bool& overrun,
                        const int32_t* cdf, int32_t maxv, int last)
{
    const uint32_t cum = x & ((1u << kScaleBits) - 1);
    // s = the last entry j < last with cdf[j] <= cum.  The symbol mapping puts the most probable
    // value (0) first, so most symbols end at s = 0 on one comparison; the others continue the
    // linear search from 1.
    const uint32_t c1 = static_cast<uint32_t>(cdf[1]);
    int s = 0;
    if (last > 1 && c1 <= cum) {
        s = 1;
        while (s + 1 < last && static_cast<uint32_t>(cdf[s + 1]) <= cum) {
            ++s;
        }
    }
    const uint32_t start = static_cast<uint32_t>(cdf[s]);
    const uint32_t freq = static_cast<uint32_t>(cdf[s + 1]) - start;
    x = freq * (x >> kScaleBits) + cum - start;
    // From a state in [2^23, 2^31) (every state a valid stream produces) at most two bytes bring
    // x back into that range (x >> 16 >= 2^7 and freq >= 1): while two bytes remain they are read
    // without per-byte bounds checks; the checked loop finishes anything else (a corrupt initial
    // state, the stream's end) exactly as byte-at-a-time reading would.
    if (x < kRansL) {
        if (!overrun && end - p >= 2) {
            x = (x << 8) | *p++;
            if (x < kRansL) {
                x = (x << 8) | *p++;
            }
        }
        while (x < kRansL && !overrun) {
            x = (x << 8) | rd_next(p, end, overrun);
        }
    }
    int32_t v = s;
    if (v == maxv) {
        int32_t b = static_cast<int32_t>(rd_bits(x, p, end, overrun));
        int32_t digits = b;
        while (b == static_cast<int32_t>(kBypassMax) && digits < 64) {
            b = static_cast<int32_t>(rd_bits(x, p, end, overrun));
            digits += b;
        }
        int32_t raw = 0;
        for (int j = 0; j < digits; ++j) {
            const int32_t d = static_cast<int32_t>(rd_bits(x, p, end, overrun));
            if (j < 16) {
                raw |= d << (2 * j);
            }
        }
        v = static_cast<int32_t>(static_cast<uint32_t>(raw) + static_cast<uint32_t>(maxv));
    }
    // 0, +1, -1, +2, -2, ... for v = 0, 1, 2, 3, 4, ...: the reference's expression (rans.cpp,
    // decode_one_symbol), kept for every v.  A corrupt stream with 16 bypass digits can set bit 31
    // of raw, and for such negative v only this form gives the reference's (and the GPU
    // decoder's) symbol; it is evaluated in 64 bits so that no input overflows.
    const int64_t w = v;
    return static_cast<int8_t>((w % 2 == 1) ? (w + 1) / 2 : -(w + 1) / 2);
}

}  // namespace

bool RansDecoderSession::begin(const uint8_t* data, int size, int ecp, std::string* err)
{
    return guarded(&fault_, err, [&] { return begin_tasks(data, size, ecp, err); });
}

bool RansDecoderSession::decode_z(const RansTables& tables, int n, int cdf_offset, int ch,
                                  int8_t* out, std::string* err)
{
    return guarded(&fault_, err, [&] { return decode_z_tasks(tables, n, cdf_offset, ch, out, err); });
}

bool RansDecoderSession::decode_y(const RansTables& tables, const uint8_t* idx, int n,
                                  int8_t* out, std::string* err)
{
    return guarded(&fault_, err, [&] { return decode_y_tasks(tables, idx, n, out, err); });
}

bool RansDecoderSession::begin_tasks(const uint8_t* data, int size, int ecp, std::string* err)
{
    ecp_ = 0;
    if (ecp < 1 || ecp > kMaxEcParallel || size < 0 || (size > 0 && data == nullptr)) {
        *err = "rANS decode: bad arguments";
        return false;
    }
    if (ecp == 1) {
        parts_[0].assign(data, data + size);
    } else {
        const int pairs = ecp / 2;
        const bool tail = (ecp % 2) != 0;
        const int noff = pairs - 1 + (tail ? 1 : 0);
        if (size < noff * 4) {
            *err = "rANS decode: stream shorter than its header";
            return false;
        }
        int32_t off[kMaxEcParallel];
        for (int k = 0; k < noff; ++k) {
            std::memcpy(&off[k], data + 4 * k, 4);
        }
        const uint8_t* pay = data + noff * 4;
        const int pay_n = size - noff * 4;
        int prev = 0;
        for (int k = 0; k < noff; ++k) {
            if (off[k] < prev || off[k] > pay_n) {
                *err = "rANS decode: inconsistent sub-stream offsets";
                return false;
            }
            prev = off[k];
        }
        for (int p = 0; p < pairs; ++p) {
            const int g0 = (p == 0) ? 0 : off[p - 1];
            const int g1 = (p < noff) ? off[p] : (tail ? off[noff - 1] : pay_n);
            parts_[2 * p].assign(pay + g0, pay + g1);
            parts_[2 * p + 1].assign(parts_[2 * p].rbegin(), parts_[2 * p].rend());
        }
        if (tail) {
            parts_[ecp - 1].assign(pay + off[noff - 1], pay + pay_n);
        }
    }
    for (int i = 0; i < ecp; ++i) {
        Reader& r = r_[i];
        r.p = parts_[i].data();
        r.end = r.p + parts_[i].size();
        r.overrun = false;
        r.x = 0;
        for (int k = 0; k < 4; ++k) {
            r.x |= static_cast<uint32_t>(rd_next(r.p, r.end, r.overrun)) << (8 * k);
        }
    }
    ecp_ = ecp;
    return true;
}

bool RansDecoderSession::decode_z_tasks(const RansTables& tables, int n, int cdf_offset, int ch,
                                        int8_t* out, std::string* err)
{
    const RansTable& tz = tables.z();
    if (ecp_ == 0 || tz.count == 0 || n < 0 || ch < 1 || cdf_offset < 0 ||
        (n > 0 && cdf_offset + ch > tz.count)) {
        *err = "rANS decode_z: bad arguments or no stream";
        return false;
    }
    run_parallel(ecp_, [&](int i) {
        Reader r = r_[i];  // a copy on this thread's stack (see Writer)
        // the table in locals (the int8 output stores may alias anything, see decode_y)
        const size_t stride = static_cast<size_t>(tz.stride);
        const int32_t* const cdf = tz.cdf.data() + static_cast<size_t>(cdf_offset) * stride;
        const int32_t* const maxv = tz.max_value.data() + cdf_offset;
        const int last = tz.stride - 1;
        int b, e;
        split(n, ecp_, i, &b, &e);
        int chn = b % ch;  // table (k % ch) + cdf_offset, the channel stepped with k
        for (int k = b; k < e; ++k) {
            out[k] = rd_symbol(r.x, r.p, r.end, r.overrun, cdf + chn * stride, maxv[chn], last);
            chn = chn + 1 == ch ? 0 : chn + 1;
        }
        r_[i] = r;
    });
    for (int i = 0; i < ecp_; ++i) {
        if (r_[i].overrun) {
            *err = "rANS decode: sub-stream ran past its bytes (truncated or corrupt stream)";
            return false;
        }
    }
    return true;
}

bool RansDecoderSession::decode_y_tasks(const RansTables& tables, const uint8_t* idx, int n,
                                        int8_t* out, std::string* err)
{
    const RansTable& ty = tables.y();
    if (ecp_ == 0 || ty.count == 0 || n < 0) {
        *err = "rANS decode_y: bad arguments or no stream";
        return false;
    }
    bool bad[kMaxEcParallel] = {false};
    run_parallel(ecp_, [&](int i) {
        Reader r = r_[i];  // a copy on this thread's stack (see Writer)
        // the table in locals: the int8 output stores may alias anything, so fields read through
        // `ty` would be reloaded after every symbol
        const int32_t* const cdf = ty.cdf.data();
        const int32_t* const maxv = ty.max_value.data();
        const size_t stride = static_cast<size_t>(ty.stride);
        const int count = ty.count;
        const int last = ty.stride - 1;
        int b, e;
        split(n, ecp_, i, &b, &e);
        for (int k = b; k < e; ++k) {
            const int t = idx[k];
            if (t >= count) {
                bad[i] = true;
                break;
            }
            out[k] = rd_symbol(r.x, r.p, r.end, r.overrun, cdf + t * stride, maxv[t], last);
        }
        r_[i] = r;
    });
    for (int i = 0; i < ecp_; ++i) {
        if (bad[i]) {
            *err = "rANS decode: y index names a CDF table out of range";
            return false;
        }
        if (r_[i].overrun) {
            *err = "rANS decode: sub-stream ran past its bytes (truncated or corrupt stream)";
            return false;
        }
    }
    return true;
}

void rans_inject_task_fault(int sub_stream)
{
    g_inject_task.store(sub_stream >= 0 && sub_stream < kMaxEcParallel ? sub_stream : -1);
}

}  // namespace dcvc
