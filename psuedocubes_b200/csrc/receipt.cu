// Host-side receipt formatting: the canonical JSON of subtile scopes, straight from the counters.
//
// A lease transcript is sha256 over, in batch order, encoded(subtile_scopes) of every batch, where
// encoded() is json.dumps(sort_keys=True, separators=(',', ':')) of the scope list with every
// integer of magnitude >= 2^53 written as a decimal string, plus a newline.  A scope is
//   {"end": str, "first": str, "group_survivors": [int...], "local_survivors": int,
//    "output_sha256": str, "valid_focused_candidates": int}
// with keys in that (sorted) order.  Building 16,384 such dicts in Python only to serialise them
// costs far more than the device work of a lease, so the bytes are written here.
#include "common.cuh"
#include <cstring>

namespace {

struct Out {
    char *p;
    uint64_t cap, len;
    bool ok;
    void put(const char *s, uint64_t n) {
        if (len + n > cap) {
            ok = false;
            return;
        }
        memcpy(p + len, s, n);
        len += n;
    }
    void str(const char *s) { put(s, strlen(s)); }
    // decimal digits of v, quoted when it is at least 2^53 and quote_large is set
    void u64(uint64_t v, bool quote_large) {
        char buf[24];
        int i = 24;
        do {
            buf[--i] = (char)('0' + v % 10);
            v /= 10;
        } while (v);
        const bool q = quote_large && (24 - i > 16 || strtoull_ge_2_53(buf + i, 24 - i));
        if (q) put("\"", 1);
        put(buf + i, (uint64_t)(24 - i));
        if (q) put("\"", 1);
    }
    // the digits (no leading zeros) denote a value >= 2^53 = 9007199254740992
    static bool strtoull_ge_2_53(const char *d, int n) {
        if (n != 16) return n > 16;
        return memcmp(d, "9007199254740992", 16) >= 0;
    }
};

}  // namespace

extern "C" int pc_scopes_json(const uint64_t *counts, uint32_t stride, uint32_t ng, uint64_t ntiles, uint64_t first,
                              uint64_t end, uint64_t width, uint32_t tiles_per_batch, const char *digests, char *out,
                              uint64_t cap, uint64_t *len) {
    *len = 0;
    if (!counts || !digests || !out || width == 0 || end <= first || tiles_per_batch == 0 || stride < ng + 3)
        return PC_INVALID;
    if ((end - first - 1) / width + 1 != ntiles) return PC_INVALID;
    const unsigned __int128 span128 = (unsigned __int128)tiles_per_batch * width;
    Out o{out, cap, 0, true};
    uint64_t t = 0, b0 = first;
    while (b0 < end && o.ok && t < ntiles) {
        const uint64_t batch_end = span128 < end - b0 ? b0 + (uint64_t)span128 : end;
        o.str("[");
        for (uint64_t v = b0; v < batch_end && o.ok && t < ntiles; ++t) {
            const uint64_t stop = batch_end - v > width ? v + width : batch_end;
            const uint64_t *c = counts + t * stride;
            if (v != b0) o.str(",");
            o.str("{\"end\":\"");
            o.u64(stop, false);
            o.str("\",\"first\":\"");
            o.u64(v, false);
            o.str("\",\"group_survivors\":[");
            for (uint32_t g = 0; g < ng; ++g) {
                if (g) o.str(",");
                o.u64(c[1 + g], true);
            }
            o.str("],\"local_survivors\":");
            o.u64(c[ng + 1], true);
            o.str(",\"output_sha256\":\"");
            o.put(digests + t * 64, 64);
            o.str("\",\"valid_focused_candidates\":");
            o.u64(c[0], true);
            o.str("}");
            v = stop;
        }
        o.str("]\n");
        b0 = batch_end;
    }
    if (!o.ok) return PC_OVERFLOW;
    if (t != ntiles) return PC_INVALID;
    *len = o.len;
    return PC_OK;
}
