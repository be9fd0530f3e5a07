// Host FASTA/FASTQ reader of the C ABI (scb_fastx_*): a plain or gzip file, read whole into
// memory, split into records in one pass (memchr over the lines) and returned as concatenated
// sequences and headers with their offsets, ready for one host batch call.  Host code only.
//
// Line rules (the reference's FASTA/FASTQ records, src/api.rs:893-915): lines end at '\n' and lose
// any trailing '\r'; a line starting with '>' or '@' opens a record whose header is the rest of
// the line ('@' opens a FASTQ record: its sequence lines run to a line starting with '+', and the
// one line after that, the qualities, is skipped); other lines extend the open record's sequence;
// lines before the first header are ignored.  A file starting with the gzip magic is inflated
// (concatenated members included).
#include <sys/stat.h>
#include <zlib.h>

#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "scb_internal.h"

namespace {

// Growable byte buffer without zero-filling (the sequences of a read set can be gigabytes).
struct Bytes {
    uint8_t* p = nullptr;
    size_t n = 0, cap = 0;
    ~Bytes() { std::free(p); }
    bool reserve(size_t want) {
        if (want <= cap) return true;
        size_t c = cap ? cap : 1 << 16;
        while (c < want) c *= 2;
        void* q = std::realloc(p, c);
        if (!q) return false;
        p = static_cast<uint8_t*>(q);
        cap = c;
        return true;
    }
    bool append(const uint8_t* src, size_t len) {
        if (!reserve(n + len)) return false;
        std::memcpy(p + n, src, len);
        n += len;
        return true;
    }
};

struct Offsets {
    uint64_t* p = nullptr;
    size_t n = 0, cap = 0;
    ~Offsets() { std::free(p); }
    bool push(uint64_t v) {
        if (n == cap) {
            const size_t c = cap ? cap * 2 : 1 << 12;
            void* q = std::realloc(p, c * sizeof(uint64_t));
            if (!q) return false;
            p = static_cast<uint64_t*>(q);
            cap = c;
        }
        p[n++] = v;
        return true;
    }
};

scb_status read_file(const char* path, Bytes& out) {
    struct stat st;
    if (::stat(path, &st) == 0 && S_ISDIR(st.st_mode)) {
        return scb::fail(SCB_ERR_FASTX_OPEN,
                         std::string("failed to open FASTA/FASTQ '") + path + "': " + std::strerror(EISDIR));
    }
    FILE* fp = std::fopen(path, "rb");
    if (!fp) {
        return scb::fail(SCB_ERR_FASTX_OPEN,
                         std::string("failed to open FASTA/FASTQ '") + path + "': " + std::strerror(errno));
    }
    unsigned char magic[2] = {0, 0};
    const size_t got = std::fread(magic, 1, 2, fp);
    const bool gz = got == 2 && magic[0] == 0x1f && magic[1] == 0x8b;
    if (!gz) {
        if (std::fseek(fp, 0, SEEK_END) != 0) {
            std::fclose(fp);
            return scb::fail_kind(SCB_ERR_IO, std::string("'") + path + "': cannot seek");
        }
        const long size = std::ftell(fp);
        std::rewind(fp);
        if (size < 0 || !out.reserve((size_t)size + 1)) {
            std::fclose(fp);
            return scb::fail_kind(SCB_ERR_IO, std::string("'") + path + "': cannot size or hold the file");
        }
        out.n = std::fread(out.p, 1, (size_t)size, fp);
        const bool bad = std::ferror(fp) != 0;
        std::fclose(fp);
        if (bad) return scb::fail_kind(SCB_ERR_IO, std::string("'") + path + "': read failed");
        return SCB_OK;
    }
    std::fclose(fp);
    gzFile gf = gzopen(path, "rb");
    if (!gf) {
        return scb::fail(SCB_ERR_FASTX_OPEN, std::string("failed to open FASTA/FASTQ '") + path + "'");
    }
    gzbuffer(gf, 1 << 20);
    constexpr unsigned kChunk = 64u << 20;
    while (true) {
        if (!out.reserve(out.n + kChunk)) {
            gzclose(gf);
            return scb::fail_kind(SCB_ERR_IO, std::string("'") + path + "': out of host memory");
        }
        const int r = gzread(gf, out.p + out.n, kChunk);
        if (r < 0) {
            int err = 0;
            const std::string msg = gzerror(gf, &err);
            gzclose(gf);
            return scb::fail_kind(SCB_ERR_IO, std::string("'") + path + "': " + msg);
        }
        if (r == 0) break;
        out.n += (size_t)r;
    }
    gzclose(gf);
    return SCB_OK;
}

}  // namespace

struct scb_fastx {
    Bytes seqs, headers;
    Offsets offsets, header_offsets;
};

extern "C" {

scb_status scb_fastx_read(const char* path, scb_fastx** out) {
    if (!path || !out) return scb::fail_kind(SCB_ERR_INTERNAL_STATE, "null argument");
    *out = nullptr;
    Bytes file;
    SCB_TRY(read_file(path, file));
    auto f = std::make_unique<scb_fastx>();
    // sequences and headers together are never longer than the file
    if (!f->seqs.reserve(file.n + 1) || !f->offsets.push(0) || !f->header_offsets.push(0)) {
        return scb::fail_kind(SCB_ERR_IO, std::string("'") + path + "': out of host memory");
    }
    bool open = false;
    int state = 0;  // 0: FASTA (or between records), 1: FASTQ sequence lines, 2: FASTQ quality line
    const uint8_t* buf = file.p;
    size_t pos = 0;
    bool ok = true;
    while (pos < file.n && ok) {
        const void* nl = std::memchr(buf + pos, '\n', file.n - pos);
        const size_t end = nl ? (size_t)(static_cast<const uint8_t*>(nl) - buf) : file.n;
        const size_t next = nl ? end + 1 : file.n;
        size_t le = end;
        while (le > pos && buf[le - 1] == '\r') le--;
        const uint8_t* line = buf + pos;
        const size_t len = le - pos;
        pos = next;
        if (state == 2) {
            state = 0;
            continue;
        }
        if (state == 1) {
            if (len && line[0] == '+') {
                state = 2;
            } else {
                ok = f->seqs.append(line, len);
            }
            continue;
        }
        if (len && (line[0] == '>' || line[0] == '@')) {
            if (open) ok = f->offsets.push(f->seqs.n) && f->header_offsets.push(f->headers.n);
            ok = ok && f->headers.append(line + 1, len - 1);
            open = true;
            state = line[0] == '@' ? 1 : 0;
        } else if (open) {
            ok = f->seqs.append(line, len);
        }
    }
    if (ok && open) ok = f->offsets.push(f->seqs.n) && f->header_offsets.push(f->headers.n);
    if (!ok) return scb::fail_kind(SCB_ERR_IO, std::string("'") + path + "': out of host memory");
    *out = f.release();
    return SCB_OK;
}

scb_status scb_fastx_sequences(const scb_fastx* f, const uint8_t** seqs, const uint64_t** offsets,
                               uint64_t* n_records) {
    if (!f || !seqs || !offsets || !n_records) return scb::fail_kind(SCB_ERR_INTERNAL_STATE, "null argument");
    *seqs = f->seqs.p;
    *offsets = f->offsets.p;
    *n_records = f->offsets.n - 1;
    return SCB_OK;
}

scb_status scb_fastx_headers(const scb_fastx* f, const uint8_t** headers, const uint64_t** header_offsets) {
    if (!f || !headers || !header_offsets) return scb::fail_kind(SCB_ERR_INTERNAL_STATE, "null argument");
    *headers = f->headers.p;
    *header_offsets = f->header_offsets.p;
    return SCB_OK;
}

void scb_fastx_free(scb_fastx* f) { delete f; }

}  // extern "C"
