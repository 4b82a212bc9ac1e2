// evxg_mux.cpp -- the packet container of the EVX ecosystem (the reference's
// evx_muxer / evx_demuxer, src/muxer.h:53-160, src/muxer.cpp), written for
// this library.  The wire layout is fixed by the reference's packed structs;
// here every field is serialised explicitly, little-endian, so the bytes do
// not depend on the host compiler's struct layout.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "evxg.h"

namespace evxg {
int fail(int code, const char *what);
}

namespace {

constexpr size_t kHeaderBytes = 10, kDescBytes = 18, kPacketBytes = 16;

void put16(uint8_t *p, uint16_t v) { p[0] = (uint8_t)v; p[1] = (uint8_t)(v >> 8); }
void put32(uint8_t *p, uint32_t v) { for (int i = 0; i < 4; i++) p[i] = (uint8_t)(v >> (8 * i)); }
void put64(uint8_t *p, uint64_t v) { for (int i = 0; i < 8; i++) p[i] = (uint8_t)(v >> (8 * i)); }
uint16_t get16(const uint8_t *p) { return (uint16_t)(p[0] | (p[1] << 8)); }
uint32_t get32(const uint8_t *p) { uint32_t v = 0; for (int i = 3; i >= 0; i--) v = (v << 8) | p[i]; return v; }
uint64_t get64(const uint8_t *p) { uint64_t v = 0; for (int i = 7; i >= 0; i--) v = (v << 8) | p[i]; return v; }

// evx_stream_descriptor (muxer.h:69-83): type, id, width, height, frame rate,
// sample rate, channels, bit depth, quality, one pad byte (zero).
void encode_desc(const evxg_stream_desc &d, uint8_t out[kDescBytes])
{
    std::memset(out, 0, kDescBytes);
    out[0] = d.stream_type;
    out[1] = d.stream_id;
    put16(out + 2, d.width);
    put16(out + 4, d.height);
    uint32_t fr;
    std::memcpy(&fr, &d.frame_rate, 4);
    put32(out + 6, fr);
    put32(out + 10, d.sample_rate);
    out[14] = d.channels;
    out[15] = d.bit_depth;
    out[16] = d.quality;
}
evxg_stream_desc decode_desc(const uint8_t in[kDescBytes])
{
    evxg_stream_desc d{};
    d.stream_type = in[0];
    d.stream_id = in[1];
    d.width = get16(in + 2);
    d.height = get16(in + 4);
    const uint32_t fr = get32(in + 6);
    std::memcpy(&d.frame_rate, &fr, 4);
    d.sample_rate = get32(in + 10);
    d.channels = in[14];
    d.bit_depth = in[15];
    d.quality = in[16];
    return d;
}

}  // namespace

struct evxg_muxer {
    FILE *f = nullptr;
    std::vector<evxg_stream_desc> streams;
    bool header_written = false;
};

struct evxg_demuxer {
    FILE *f = nullptr;
    std::vector<evxg_stream_desc> streams;
};

using evxg::fail;

extern "C" {

int evxg_muxer_open(const char *path, evxg_muxer **out)
{
    if (!path || !out) return fail(EVXG_ERROR_INVALIDARG, "evxg_muxer_open: null argument");
    *out = nullptr;
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(EVXG_ERROR_IO_FAILURE, "evxg_muxer_open: cannot create the file");
    evxg_muxer *m = new (std::nothrow) evxg_muxer();
    if (!m) {
        std::fclose(f);
        return fail(EVXG_ERROR_OUTOFMEMORY, "evxg_muxer_open: host allocation");
    }
    m->f = f;
    *out = m;
    return EVXG_SUCCESS;
}

static int add_stream(evxg_muxer *m, evxg_stream_desc d, uint8_t *id, const char *who)
{
    if (!m || !id || m->header_written) return fail(EVXG_ERROR_INVALIDARG, who);
    if (m->streams.size() >= 255) return fail(EVXG_ERROR_CAPACITY_LIMIT, who);
    d.stream_id = (uint8_t)m->streams.size();
    m->streams.push_back(d);
    *id = d.stream_id;
    return EVXG_SUCCESS;
}

int evxg_muxer_add_video_stream(evxg_muxer *m, uint16_t width, uint16_t height, float frame_rate, uint8_t *stream_id)
{
    evxg_stream_desc d{};
    d.stream_type = EVXG_STREAM_TYPE_VIDEO;
    d.width = width;
    d.height = height;
    d.frame_rate = frame_rate;
    return add_stream(m, d, stream_id, "evxg_muxer_add_video_stream: null argument or header already written");
}

int evxg_muxer_add_audio_stream(evxg_muxer *m, uint32_t sample_rate, uint8_t channels, uint8_t bit_depth,
                                uint8_t quality, uint8_t *stream_id)
{
    evxg_stream_desc d{};
    d.stream_type = EVXG_STREAM_TYPE_AUDIO;
    d.sample_rate = sample_rate;
    d.channels = channels;
    d.bit_depth = bit_depth;
    d.quality = quality;
    return add_stream(m, d, stream_id, "evxg_muxer_add_audio_stream: null argument or header already written");
}

int evxg_muxer_write_header(evxg_muxer *m)
{
    if (!m || !m->f || m->header_written) return fail(EVXG_ERROR_NOT_READY, "evxg_muxer_write_header: not open or written");
    std::vector<uint8_t> b(kHeaderBytes + m->streams.size() * kDescBytes);
    std::memcpy(b.data(), "EVX3", 4);
    put32(b.data() + 4, (uint32_t)b.size());   // header size: the header and its descriptors
    b[8] = 1;                                  // version
    b[9] = (uint8_t)m->streams.size();
    for (size_t i = 0; i < m->streams.size(); i++) encode_desc(m->streams[i], b.data() + kHeaderBytes + i * kDescBytes);
    if (std::fwrite(b.data(), 1, b.size(), m->f) != b.size()) return fail(EVXG_ERROR_IO_FAILURE, "evxg_muxer_write_header");
    m->header_written = true;
    return EVXG_SUCCESS;
}

int evxg_muxer_write_packet(evxg_muxer *m, uint8_t stream_id, uint8_t stream_type, uint64_t timestamp_us,
                            const void *payload, uint32_t size)
{
    if (!m || !m->f || !m->header_written || !payload || !size)
        return fail(EVXG_ERROR_INVALIDARG, "evxg_muxer_write_packet: not ready, or an empty payload");
    uint8_t h[kPacketBytes];
    h[0] = 'E';
    h[1] = 'P';
    h[2] = stream_id;
    h[3] = stream_type;
    put64(h + 4, timestamp_us);
    put32(h + 12, size);
    if (std::fwrite(h, 1, kPacketBytes, m->f) != kPacketBytes || std::fwrite(payload, 1, size, m->f) != size)
        return fail(EVXG_ERROR_IO_FAILURE, "evxg_muxer_write_packet");
    return EVXG_SUCCESS;
}

int evxg_muxer_close(evxg_muxer *m)
{
    if (!m) return EVXG_ERROR_INVALIDARG;
    const int rc = (m->f && std::fclose(m->f) != 0) ? fail(EVXG_ERROR_IO_FAILURE, "evxg_muxer_close") : EVXG_SUCCESS;
    delete m;
    return rc;
}

int evxg_demuxer_open(const char *path, evxg_demuxer **out)
{
    if (!path || !out) return fail(EVXG_ERROR_INVALIDARG, "evxg_demuxer_open: null argument");
    *out = nullptr;
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(EVXG_ERROR_IO_FAILURE, "evxg_demuxer_open: cannot open the file");
    uint8_t h[kHeaderBytes];
    if (std::fread(h, 1, kHeaderBytes, f) != kHeaderBytes) {
        std::fclose(f);
        return fail(EVXG_ERROR_IO_FAILURE, "evxg_demuxer_open: short header");
    }
    if (std::memcmp(h, "EVX3", 4) != 0) {
        std::fclose(f);
        return fail(EVXG_ERROR_INVALID_RESOURCE, "evxg_demuxer_open: not an EVX3 container");
    }
    evxg_demuxer *d = new (std::nothrow) evxg_demuxer();
    if (!d) {
        std::fclose(f);
        return fail(EVXG_ERROR_OUTOFMEMORY, "evxg_demuxer_open: host allocation");
    }
    d->f = f;
    for (int i = 0; i < h[9]; i++) {   // the descriptors follow the header (muxer.cpp reads stream_count of them)
        uint8_t b[kDescBytes];
        if (std::fread(b, 1, kDescBytes, f) != kDescBytes) {
            evxg_demuxer_close(d);
            return fail(EVXG_ERROR_IO_FAILURE, "evxg_demuxer_open: short stream descriptor");
        }
        d->streams.push_back(decode_desc(b));
    }
    *out = d;
    return EVXG_SUCCESS;
}

uint32_t evxg_demuxer_stream_count(const evxg_demuxer *d) { return d ? (uint32_t)d->streams.size() : 0; }

int evxg_demuxer_stream(const evxg_demuxer *d, uint32_t index, evxg_stream_desc *out)
{
    if (!d || !out || index >= d->streams.size()) return fail(EVXG_ERROR_INVALID_INDEX, "evxg_demuxer_stream: bad index");
    *out = d->streams[index];
    return EVXG_SUCCESS;
}

int evxg_demuxer_read_packet(evxg_demuxer *d, uint8_t *stream_id, uint8_t *stream_type, uint64_t *timestamp_us,
                             uint8_t *payload, uint32_t capacity, uint32_t *size)
{
    if (!d || !d->f || !size) return fail(EVXG_ERROR_INVALIDARG, "evxg_demuxer_read_packet: null argument");
    uint8_t h[kPacketBytes];
    const size_t got = std::fread(h, 1, kPacketBytes, d->f);
    if (got != kPacketBytes) {
        if (got == 0 && std::feof(d->f)) return EVXG_ERROR_OPERATION_COMPLETED;
        return fail(EVXG_ERROR_IO_FAILURE, "evxg_demuxer_read_packet: short packet header");
    }
    if (h[0] != 'E' || h[1] != 'P') return fail(EVXG_ERROR_INVALID_RESOURCE, "evxg_demuxer_read_packet: bad packet magic");
    const uint32_t n = get32(h + 12);
    *size = n;
    if (n > capacity || (n && !payload)) {   // leave the packet for a call with a larger buffer
        std::fseek(d->f, -(long)kPacketBytes, SEEK_CUR);
        return EVXG_ERROR_CAPACITY_LIMIT;
    }
    if (n && std::fread(payload, 1, n, d->f) != n)
        return fail(EVXG_ERROR_IO_FAILURE, "evxg_demuxer_read_packet: short payload");
    if (stream_id) *stream_id = h[2];
    if (stream_type) *stream_type = h[3];
    if (timestamp_us) *timestamp_us = get64(h + 4);
    return EVXG_SUCCESS;
}

int evxg_demuxer_close(evxg_demuxer *d)
{
    if (!d) return EVXG_ERROR_INVALIDARG;
    if (d->f) std::fclose(d->f);
    delete d;
    return EVXG_SUCCESS;
}

}  // extern "C"
