/*
 * ORACLE (test infrastructure only; never linked into the product).
 *
 * Plain, single-threaded C restatement of the reference's MLCodec rANS coder and its
 * multi-stream container.  Used by tests/ and by bench.py's CPU baseline as the checker for
 * the product coder (dcvc_b200/csrc/rans_coder.cpp).  Pinned against the reference compiled
 * from its own sources (oracle/_ref/librans_ref.so, built by oracle/Makefile) and against the
 * committed golden streams under tests/golden/.
 *
 * Reference anchors (paths inside the reference project):
 *   constants                     src/cpp/py_rans/rans.cpp:13-19
 *   RansEncPut / RansEncPutBits   src/cpp/py_rans/rans.cpp:76-102
 *   RansDecAdvance/GetBits/Init   src/cpp/py_rans/rans.cpp:29-66
 *   decode_one_symbol             src/cpp/py_rans/rans.cpp:104-142
 *   encode_one_symbol             src/cpp/py_rans/rans.cpp:144-181
 *   encode_y/z_internal           src/cpp/py_rans/rans.cpp:239-294 (backward over symbols)
 *   decode_y/z_internal           src/cpp/py_rans/rans.cpp:417-463
 *   sub-stream split              src/cpp/py_rans/py_rans.cpp:104-135, 287-337
 *   container merge               src/cpp/py_rans/py_rans.cpp:16-33, 156-249
 *   container split               src/cpp/py_rans/py_rans.cpp:412-492
 *   pmf_to_quantized_cdf          src/cpp/py_rans/py_rans.cpp:35-94
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define SCALE_BITS 16
#define L_BITS 23
#define RANS_L (1u << L_BITS)
#define RENORM_SHIFT (L_BITS - SCALE_BITS + 8)
#define BYPASS_BITS 2
#define BYPASS_MAX ((1u << BYPASS_BITS) - 1u)

/* ---------------------------------------------------------------- pmf -> cdf */

int oracle_pmf_to_quantized_cdf(const float* pmf, int n, uint32_t* cdf)
{
    const uint32_t prob_max = 1u << 16;
    int m = n + 1;
    cdf[0] = 0;
    for (int i = 0; i < n; i++) {
        /* float * float, then + 0.5 in double, truncated to uint32 */
        float prod = pmf[i] * (float)prob_max;
        cdf[i + 1] = (uint32_t)((double)prod + 0.5);
    }
    int total = 0; /* std::accumulate with an int initial value */
    for (int i = 0; i < m; i++) total += (int)cdf[i];
    for (int i = 0; i < m; i++) {
        cdf[i] = (uint32_t)(((uint64_t)prob_max * cdf[i]) / (uint32_t)total);
    }
    for (int i = 1; i < m; i++) cdf[i] += cdf[i - 1];
    cdf[m - 1] = prob_max;
    for (int i = 0; i < m - 1; i++) {
        if (cdf[i] + 1 > cdf[i + 1]) {
            uint32_t best_freq = ~0u;
            int best = -1;
            for (int j = 0; j < m - 1; j++) {
                uint32_t f = cdf[j + 1] - cdf[j];
                if (f >= 2 && f < best_freq) {
                    best_freq = f;
                    best = j;
                }
            }
            if (best < 0) return -1;
            if (best < i) {
                for (int j = best + 1; j <= i; j++) cdf[j] -= 1;
            } else {
                for (int j = i + 1; j <= best; j++) cdf[j] += 1;
            }
        }
    }
    return m;
}

/* ---------------------------------------------------------------- one stream */

typedef struct {
    uint8_t* buf; /* bytes are written backwards from buf + cap */
    int cap;
    int pos; /* index of the first valid byte */
    uint32_t x;
} enc_t;

static int enc_byte(enc_t* e, uint8_t b)
{
    if (e->pos == 0) return -1;
    e->buf[--e->pos] = b;
    return 0;
}

static int enc_put(enc_t* e, uint32_t start, uint32_t freq)
{
    uint32_t x_max = freq << RENORM_SHIFT;
    while (e->x >= x_max) {
        if (enc_byte(e, (uint8_t)(e->x & 0xff))) return -1;
        e->x >>= 8;
    }
    e->x = ((e->x / freq) << SCALE_BITS) + (e->x % freq) + start;
    return 0;
}

static int enc_bits(enc_t* e, uint32_t v)
{
    const uint32_t x_max = (1u << (SCALE_BITS - BYPASS_BITS)) << RENORM_SHIFT;
    while (e->x >= x_max) {
        if (enc_byte(e, (uint8_t)(e->x & 0xff))) return -1;
        e->x >>= 8;
    }
    e->x = (e->x << BYPASS_BITS) | v;
    return 0;
}

/* cdf: one table of `stride` int32 entries; maxv = cdf_length - 2 */
static int enc_symbol(enc_t* e, int32_t s, const int32_t* cdf, int32_t maxv)
{
    int32_t v = abs(s) * 2 - (s > 0);
    if (v >= maxv) {
        uint32_t raw = (uint32_t)(v - maxv);
        uint32_t bins[64];
        int nb = 0;
        int nbp = 0;
        while ((raw >> (nbp * BYPASS_BITS)) != 0) nbp++;
        int32_t cnt = nbp;
        while (cnt >= (int32_t)BYPASS_MAX) {
            bins[nb++] = BYPASS_MAX;
            cnt -= BYPASS_MAX;
        }
        bins[nb++] = (uint32_t)cnt;
        for (int j = 0; j < nbp; j++) bins[nb++] = (raw >> (j * BYPASS_BITS)) & BYPASS_MAX;
        for (int j = nb - 1; j >= 0; j--) {
            if (enc_bits(e, bins[j])) return -1;
        }
        v = maxv;
    }
    uint32_t start = (uint16_t)cdf[v];
    uint32_t freq = (uint16_t)(cdf[v + 1] - cdf[v]);
    return enc_put(e, start, freq);
}

static int enc_flush(enc_t* e)
{
    for (int k = 3; k >= 0; k--) {
        if (enc_byte(e, (uint8_t)(e->x >> (8 * k)))) return -1;
    }
    return 0;
}

typedef struct {
    const uint8_t* p;
    const uint8_t* end;
    uint32_t x;
    int overrun;
} dec_t;

static uint8_t dec_byte(dec_t* d)
{
    if (d->p >= d->end) {
        d->overrun = 1;
        return 0;
    }
    return *d->p++;
}

static void dec_init(dec_t* d, const uint8_t* p, int n)
{
    d->p = p;
    d->end = p + n;
    d->overrun = 0;
    uint32_t x = 0;
    for (int k = 0; k < 4; k++) x |= (uint32_t)dec_byte(d) << (8 * k);
    d->x = x;
}

static uint32_t dec_bits(dec_t* d)
{
    uint32_t v = d->x & BYPASS_MAX;
    d->x >>= BYPASS_BITS;
    if (d->x < RANS_L) d->x = (d->x << 8) | dec_byte(d);
    return v;
}

static int8_t dec_symbol(dec_t* d, const int32_t* cdf, int32_t maxv)
{
    uint32_t cum = d->x & ((1u << SCALE_BITS) - 1);
    int s = 1;
    while ((uint32_t)cdf[s] <= cum) s++;
    s--;
    uint32_t start = (uint32_t)cdf[s];
    uint32_t freq = (uint32_t)(cdf[s + 1] - cdf[s]);
    d->x = freq * (d->x >> SCALE_BITS) + (d->x & ((1u << SCALE_BITS) - 1)) - start;
    while (d->x < RANS_L) d->x = (d->x << 8) | dec_byte(d);
    int32_t v = s;
    if (v == maxv) {
        int32_t b = (int32_t)dec_bits(d);
        int32_t nbp = b;
        while (b == (int32_t)BYPASS_MAX) {
            b = (int32_t)dec_bits(d);
            nbp += b;
        }
        int32_t raw = 0;
        /* digits past the 16th would shift past bit 31 (undefined in the reference's C++, which
         * a valid stream never reaches: |v| <= 256); they are read and dropped */
        for (int j = 0; j < nbp; j++) {
            uint32_t digit = dec_bits(d);
            if (j < 16) raw = (int32_t)((uint32_t)raw | (digit << (j * BYPASS_BITS)));
        }
        v = (int32_t)((uint32_t)raw + (uint32_t)maxv);
    }
    {
        int64_t w = v;
        return (int8_t)((w % 2 == 1) ? (w + 1) / 2 : -(w + 1) / 2);
    }
}

/* ---------------------------------------------------------------- container */

static int common_tail_bytes(const uint8_t* a, int na, const uint8_t* b, int nb)
{
    int lim = na < nb ? na : nb;
    if (lim > 8) lim = 8;
    int k = 0;
    for (int i = 0; i < lim; i++) {
        if (a[na - 1 - i] != 0 || b[nb - 1 - i] != 0) break;
        k++;
    }
    if (k == 0 && a[na - 1] == b[nb - 1]) k = 1;
    return k;
}

/* Encodes `n_seg` y segments (concatenated in y_sym, lengths y_counts, in coding order) then the
 * z symbols into `ecp` sub-streams and merges them.  Every segment is split evenly over the
 * sub-streams and each sub-stream codes its slices back to front, segment after segment (one
 * encode_y call per segment, py_rans.cpp:104-135).  Returns the number of bytes written, -1 on
 * a capacity problem, -2 on bad arguments. */
int oracle_encode_segments(const int32_t* cdf_z, const int32_t* len_z, int z_stride,
                           const int32_t* cdf_y, const int32_t* len_y, int y_stride,
                           const int16_t* y_sym, const int* y_counts, int n_seg,
                           const int8_t* z_sym, int n_z, int z_cdf_offset, int z_ch, int ecp,
                           uint8_t* out, int out_cap)
{
    if (ecp < 1 || ecp > 8 || z_ch < 1 || n_seg < 0) return -2;
    int n_y = 0;
    for (int g = 0; g < n_seg; g++) {
        if (y_counts[g] < 0) return -2;
        n_y += y_counts[g];
    }
    enc_t e[8];
    int rc = 0;
    for (int i = 0; i < ecp; i++) {
        e[i].cap = (n_y / ecp + 8 * n_seg + n_z / ecp + 8) * 4 + 4;
        e[i].buf = (uint8_t*)malloc((size_t)e[i].cap + 1);
        e[i].pos = e[i].cap;
        e[i].x = RANS_L;
    }
    for (int i = 0; i < ecp && rc == 0; i++) {
        const int16_t* seg = y_sym;
        for (int g = 0; g < n_seg && rc == 0; g++) {
            int ng = y_counts[g];
            int sy = ng / ecp;
            int y0 = sy * i;
            int y1 = (i < ecp - 1) ? y0 + sy : ng;
            for (int k = y1 - 1; k >= y0 && rc == 0; k--) {
                int16_t c = seg[k];
                int idx = c & 0xff;
                int32_t s = (int8_t)(c >> 8);
                rc = enc_symbol(&e[i], s, cdf_y + (size_t)idx * y_stride, len_y[idx] - 2);
            }
            seg += ng;
        }
        int sz = n_z / ecp;
        int z0 = sz * i;
        int z1 = (i < ecp - 1) ? z0 + sz : n_z;
        for (int k = z1 - 1; k >= z0 && rc == 0; k--) {
            int t = (k % z_ch) + z_cdf_offset;
            rc = enc_symbol(&e[i], z_sym[k], cdf_z + (size_t)t * z_stride, len_z[t] - 2);
        }
        if (rc == 0) rc = enc_flush(&e[i]);
    }
    int total = -1;
    if (rc == 0) {
        const uint8_t* s[8];
        int n[8];
        for (int i = 0; i < ecp; i++) {
            s[i] = e[i].buf + e[i].pos;
            n[i] = e[i].cap - e[i].pos;
        }
        if (ecp == 1) {
            total = n[0];
            if (total <= out_cap) memcpy(out, s[0], (size_t)n[0]);
            else total = -1;
        } else {
            int pairs = ecp / 2;
            int tail = ecp % 2;
            int same[4], gsz[4];
            for (int p = 0; p < pairs; p++) {
                same[p] = common_tail_bytes(s[2 * p], n[2 * p], s[2 * p + 1], n[2 * p + 1]);
                gsz[p] = n[2 * p] + n[2 * p + 1] - same[p];
            }
            int noff = pairs - 1 + tail;
            total = noff * 4;
            for (int p = 0; p < pairs; p++) total += gsz[p];
            if (tail) total += n[ecp - 1];
            if (total > out_cap) {
                total = -1;
            } else {
                /* offset k = bytes of groups 0..k; with a tail the last one is the tail start */
                int cum = gsz[0];
                for (int k = 0; k < noff; k++) {
                    int32_t v = cum;
                    memcpy(out + 4 * k, &v, 4);
                    if (k + 1 < pairs) cum += gsz[k + 1];
                }
                int pos = noff * 4;
                for (int p = 0; p < pairs; p++) {
                    const uint8_t* a = s[2 * p];
                    const uint8_t* b = s[2 * p + 1];
                    memcpy(out + pos, a, (size_t)n[2 * p]);
                    int nb = n[2 * p + 1] - same[p];
                    for (int j = 0; j < nb; j++) out[pos + n[2 * p] + j] = b[nb - 1 - j];
                    pos += gsz[p];
                }
                if (tail) memcpy(out + pos, s[ecp - 1], (size_t)n[ecp - 1]);
            }
        }
    }
    for (int i = 0; i < ecp; i++) free(e[i].buf);
    return total;
}

/* One y segment then z (the video model's payload). */
int oracle_encode(const int32_t* cdf_z, const int32_t* len_z, int z_stride, const int32_t* cdf_y,
                  const int32_t* len_y, int y_stride, const int16_t* y_sym, int n_y,
                  const int8_t* z_sym, int n_z, int z_cdf_offset, int z_ch, int ecp, uint8_t* out,
                  int out_cap)
{
    return oracle_encode_segments(cdf_z, len_z, z_stride, cdf_y, len_y, y_stride, y_sym, &n_y, 1,
                                  z_sym, n_z, z_cdf_offset, z_ch, ecp, out, out_cap);
}

/* Incremental decoder over one container: split once (py_rans.cpp:412-492), then segments are
 * decoded in the reverse order of encoding, each split evenly over the sub-streams. */
typedef struct {
    int ecp;
    uint8_t* part[8];
    int psz[8];
    dec_t d[8];
} odec_t;

void oracle_dec_close(void* h)
{
    odec_t* o = (odec_t*)h;
    if (o == NULL) return;
    for (int i = 0; i < 8; i++) free(o->part[i]);
    free(o);
}

/* NULL on a malformed container or bad arguments. */
void* oracle_dec_open(const uint8_t* stream, int size, int ecp)
{
    if (ecp < 1 || ecp > 8 || size < 0) return NULL;
    odec_t* o = (odec_t*)calloc(1, sizeof(odec_t));
    if (o == NULL) return NULL;
    o->ecp = ecp;
    if (ecp == 1) {
        o->part[0] = (uint8_t*)malloc((size_t)size + 1);
        memcpy(o->part[0], stream, (size_t)size);
        o->psz[0] = size;
    } else {
        int pairs = ecp / 2;
        int tail = ecp % 2;
        int noff = pairs - 1 + tail;
        int off[4];
        if (size < noff * 4) {
            oracle_dec_close(o);
            return NULL;
        }
        for (int k = 0; k < noff; k++) memcpy(&off[k], stream + 4 * k, 4);
        const uint8_t* pay = stream + noff * 4;
        int pay_n = size - noff * 4;
        for (int p = 0; p < pairs; p++) {
            int g0 = (p == 0) ? 0 : off[p - 1];
            int g1;
            if (p < noff) g1 = off[p];
            else g1 = tail ? off[noff - 1] : pay_n;
            if (noff == 0) g1 = pay_n;
            if (g0 < 0 || g1 > pay_n || g1 < g0) {
                oracle_dec_close(o);
                return NULL;
            }
            int gs = g1 - g0;
            o->part[2 * p] = (uint8_t*)malloc((size_t)gs + 1);
            o->part[2 * p + 1] = (uint8_t*)malloc((size_t)gs + 1);
            memcpy(o->part[2 * p], pay + g0, (size_t)gs);
            for (int j = 0; j < gs; j++) o->part[2 * p + 1][j] = pay[g1 - 1 - j];
            o->psz[2 * p] = o->psz[2 * p + 1] = gs;
        }
        if (tail) {
            int t0 = off[noff - 1];
            int ts = pay_n - t0;
            if (t0 < 0 || ts < 0) {
                oracle_dec_close(o);
                return NULL;
            }
            o->part[ecp - 1] = (uint8_t*)malloc((size_t)ts + 1);
            memcpy(o->part[ecp - 1], pay + t0, (size_t)ts);
            o->psz[ecp - 1] = ts;
        }
    }
    for (int i = 0; i < ecp; i++) dec_init(&o->d[i], o->part[i], o->psz[i]);
    return o;
}

/* 0, or -3 if a sub-stream ran past its bytes. */
int oracle_dec_z(void* h, const int32_t* cdf_z, const int32_t* len_z, int z_stride, int n_z,
                 int z_cdf_offset, int z_ch, int8_t* z_out)
{
    odec_t* o = (odec_t*)h;
    int rc = 0;
    for (int i = 0; i < o->ecp; i++) {
        int sz = n_z / o->ecp;
        int z0 = sz * i;
        int z1 = (i < o->ecp - 1) ? z0 + sz : n_z;
        for (int k = z0; k < z1; k++) {
            int t = (k % z_ch) + z_cdf_offset;
            z_out[k] = dec_symbol(&o->d[i], cdf_z + (size_t)t * z_stride, len_z[t] - 2);
        }
        if (o->d[i].overrun) rc = -3;
    }
    return rc;
}

int oracle_dec_y(void* h, const int32_t* cdf_y, const int32_t* len_y, int y_stride,
                 const uint8_t* y_idx, int n_y, int8_t* y_out)
{
    odec_t* o = (odec_t*)h;
    int rc = 0;
    for (int i = 0; i < o->ecp; i++) {
        int sy = n_y / o->ecp;
        int y0 = sy * i;
        int y1 = (i < o->ecp - 1) ? y0 + sy : n_y;
        for (int k = y0; k < y1; k++) {
            int idx = y_idx[k];
            y_out[k] = dec_symbol(&o->d[i], cdf_y + (size_t)idx * y_stride, len_y[idx] - 2);
        }
        if (o->d[i].overrun) rc = -3;
    }
    return rc;
}

/* Decodes z then y from a container made by oracle_encode.  Returns 0, -2 on bad arguments,
 * -3 if a sub-stream ran past its bytes. */
int oracle_decode(const int32_t* cdf_z, const int32_t* len_z, int z_stride, const int32_t* cdf_y,
                  const int32_t* len_y, int y_stride, const uint8_t* stream, int size,
                  const uint8_t* y_idx, int n_y, int n_z, int z_cdf_offset, int z_ch, int ecp,
                  int8_t* y_out, int8_t* z_out)
{
    if (z_ch < 1) return -2;
    void* h = oracle_dec_open(stream, size, ecp);
    if (h == NULL) return -2;
    int rc = oracle_dec_z(h, cdf_z, len_z, z_stride, n_z, z_cdf_offset, z_ch, z_out);
    int rc2 = oracle_dec_y(h, cdf_y, len_y, y_stride, y_idx, n_y, y_out);
    oracle_dec_close(h);
    return rc != 0 ? rc : rc2;
}
