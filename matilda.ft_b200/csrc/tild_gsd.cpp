// tild_gsd.cpp -- GSD 2.0 container writer (layout in tild_gsd.h).
#include <cstdio>

#include "tild_gsd.h"

#include <algorithm>
#include <cstring>

#include "tild_b200.h"
#include "tild_box.h"

namespace tild {

namespace {
constexpr uint64_t kMagic = 0x65DF65DF65DF65DFull;
constexpr size_t kHeaderBytes = 256, kEntryBytes = 32, kNameUnit = 64;
constexpr uint64_t kInitialIndex = 128, kInitialNameBytes = 1024;

void put(std::FILE *f, uint64_t at, const void *p, size_t n, const std::string &path)
{
    if (n == 0) return;
    if (std::fseek(f, (long)at, SEEK_SET) != 0 || std::fwrite(p, 1, n, f) != n)
        fail(TILD_ERR_IO, "GSD write failed: " + path);
}

void zeros(std::FILE *f, uint64_t at, uint64_t n, const std::string &path)
{
    std::vector<char> z((size_t)std::min<uint64_t>(n, 1 << 20), 0);
    while (n > 0) {
        const size_t k = (size_t)std::min<uint64_t>(n, z.size());
        put(f, at, z.data(), k, path);
        at += k;
        n -= k;
    }
}

void packEntry(char *o, uint64_t frame, uint64_t N, int64_t loc, uint32_t M, uint16_t id, uint8_t type, uint8_t flags)
{
    std::memcpy(o, &frame, 8);
    std::memcpy(o + 8, &N, 8);
    std::memcpy(o + 16, &loc, 8);
    std::memcpy(o + 24, &M, 4);
    std::memcpy(o + 28, &id, 2);
    o[30] = (char)type;
    o[31] = (char)flags;
}
}  // namespace

size_t gsd_type_size(GsdType t)
{
    switch (t) {
        case GSD_U8: case GSD_I8: return 1;
        case GSD_U16: case GSD_I16: return 2;
        case GSD_U32: case GSD_I32: case GSD_F32: return 4;
        case GSD_U64: case GSD_I64: case GSD_F64: return 8;
    }
    return 0;
}

void GsdWriter::writeHeader(std::FILE *f) const
{
    char h[kHeaderBytes];
    std::memset(h, 0, sizeof h);
    const uint32_t fileVersion = version(2, 0);
    std::memcpy(h, &kMagic, 8);
    std::memcpy(h + 8, &indexLoc_, 8);
    std::memcpy(h + 16, &indexCap_, 8);
    std::memcpy(h + 24, &nameLoc_, 8);
    std::memcpy(h + 32, &nameCap_, 8);
    std::memcpy(h + 40, &schemaVersion_, 4);
    std::memcpy(h + 44, &fileVersion, 4);
    std::strncpy(h + 48, application_.c_str(), 63);
    std::strncpy(h + 112, schema_.c_str(), 63);
    put(f, 0, h, sizeof h, path_);
}

void GsdWriter::create(const std::string &path, const char *application, const char *schema, uint32_t schema_version)
{
    path_ = path;
    application_ = application;
    schema_ = schema;
    schemaVersion_ = schema_version;
    names_.clear();
    namesWritten_ = 0;
    index_.clear();
    pending_.clear();
    frame_ = 0;
    indexLoc_ = kHeaderBytes;
    indexCap_ = kInitialIndex;
    nameLoc_ = indexLoc_ + kEntryBytes * indexCap_;
    nameCap_ = kInitialNameBytes / kNameUnit;
    fileSize_ = nameLoc_ + kInitialNameBytes;
    std::FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) {
        path_.clear();
        fail(TILD_ERR_IO, "Failed to create GSD file " + path);
    }
    writeHeader(f);
    zeros(f, indexLoc_, fileSize_ - indexLoc_, path_);
    std::fclose(f);
}

void GsdWriter::chunk(const char *name, GsdType type, uint64_t N, uint32_t M, const void *data)
{
    if (!isOpen()) fail(TILD_ERR_STATE, "GSD file not created");
    if (M == 0 || gsd_type_size(type) == 0) fail(TILD_ERR_ARG, std::string("bad GSD chunk ") + name);
    const auto it = std::find(names_.begin(), names_.end(), std::string(name));
    uint16_t id;
    if (it == names_.end()) {
        if (names_.size() >= 0xFFFF) fail(TILD_ERR_ARG, "GSD namelist full");
        id = (uint16_t)names_.size();
        names_.push_back(name);
    } else {
        id = (uint16_t)(it - names_.begin());
    }
    Pending p{id, type, N, M, {}};
    const size_t bytes = (size_t)(N * M * gsd_type_size(type));
    p.bytes.assign(static_cast<const char *>(data), static_cast<const char *>(data) + bytes);
    pending_.push_back(std::move(p));
}

void GsdWriter::endFrame()
{
    if (!isOpen()) fail(TILD_ERR_STATE, "GSD file not created");
    std::FILE *f = std::fopen(path_.c_str(), "r+b");
    if (!f) fail(TILD_ERR_IO, "Failed to open GSD file " + path_);
    // chunk data at the end of the file, in the order written
    std::vector<Entry> add;
    for (const Pending &p : pending_) {
        add.push_back({frame_, p.N, (int64_t)fileSize_, p.M, p.id, (uint8_t)p.type, 0});
        put(f, fileSize_, p.bytes.data(), p.bytes.size(), path_);
        fileSize_ += p.bytes.size();
    }
    pending_.clear();
    // names: rewrite the whole list, moved to the end at double size when it outgrows its region
    if (names_.size() > namesWritten_) {
        std::vector<char> list;
        for (const std::string &s : names_) list.insert(list.end(), s.c_str(), s.c_str() + s.size() + 1);
        uint64_t cap = nameCap_;
        while (cap * kNameUnit < list.size() + 1) cap *= 2;   // keep a terminating 0 byte
        if (cap != nameCap_) {
            nameLoc_ = fileSize_;
            nameCap_ = cap;
            fileSize_ += cap * kNameUnit;
            zeros(f, nameLoc_, cap * kNameUnit, path_);
        }
        put(f, nameLoc_, list.data(), list.size(), path_);
        namesWritten_ = names_.size();
    }
    // index: this frame's entries sorted by name id after the earlier frames' entries
    std::stable_sort(add.begin(), add.end(), [](const Entry &a, const Entry &b) { return a.id < b.id; });
    const size_t first = index_.size();
    index_.insert(index_.end(), add.begin(), add.end());
    uint64_t cap = indexCap_;
    while (cap <= index_.size() || cap <= frame_) cap *= 2;
    size_t from = first;
    if (cap != indexCap_) {   // move the index to the end of the file
        indexLoc_ = fileSize_;
        indexCap_ = cap;
        fileSize_ += cap * kEntryBytes;
        zeros(f, indexLoc_, cap * kEntryBytes, path_);
        from = 0;
    }
    std::vector<char> buf((index_.size() - from) * kEntryBytes);
    for (size_t k = from; k < index_.size(); k++) {
        const Entry &e = index_[k];
        packEntry(buf.data() + (k - from) * kEntryBytes, e.frame, e.N, e.location, e.M, e.id, e.type, e.flags);
    }
    put(f, indexLoc_ + from * kEntryBytes, buf.data(), buf.size(), path_);
    writeHeader(f);
    if (std::fclose(f) != 0) fail(TILD_ERR_IO, "GSD write failed: " + path_);
    frame_++;
}

}  // namespace tild
