// tild_gsd.h -- writer for the GSD 2.0 container (the HOOMD-blue project's "General
// Simulation Data" file format), the trajectory format PS_Box::writeGSDtraj produces
// (PS_Box_gsdUtils.cu:14-168 through the vendored gsd.c).
//
// Layout written here, as the format specifies it:
//   [0, 256)            header: magic 0x65DF65DF65DF65DF, index location, index capacity
//                       (entries), namelist location, namelist capacity (units of 64 bytes),
//                       schema version, file version 2.0, application[64], schema[64],
//                       reserved[80]
//   index               capacity x 32-byte entries {u64 frame, u64 N, i64 location, u32 M,
//                       u16 name id, u8 type, u8 flags}, sorted by (frame, id); the first
//                       entry with location 0 ends the list; every frame < capacity
//   namelist            NUL-terminated names packed back to back, id = position in the list;
//                       an empty name (and the region's last byte) is 0
//   chunk data          appended to the end of the file in the order written
// The index and namelist start right after the header (128 entries, 1024 bytes) and are
// moved to the end of the file, at double the size, when a frame outgrows them.
#pragma once
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

namespace tild {

enum GsdType : uint8_t {
    GSD_U8 = 1, GSD_U16, GSD_U32, GSD_U64, GSD_I8, GSD_I16, GSD_I32, GSD_I64, GSD_F32, GSD_F64
};

class GsdWriter {
public:
    // Truncate or create `path` and write an empty header, index and namelist.
    void create(const std::string &path, const char *application, const char *schema, uint32_t schema_version);
    bool isOpen() const { return !path_.empty(); }
    // Add a chunk (N rows x M columns of `type`) to the current frame; the bytes are copied.
    void chunk(const char *name, GsdType type, uint64_t N, uint32_t M, const void *data);
    // Append the frame's chunk data, names and index entries, then rewrite the header.
    void endFrame();
    uint64_t frames() const { return frame_; }
    static uint32_t version(unsigned major, unsigned minor) { return (uint32_t)major << 16 | minor; }

private:
    struct Entry {
        uint64_t frame, N;
        int64_t location;
        uint32_t M;
        uint16_t id;
        uint8_t type, flags;
    };
    struct Pending {
        uint16_t id;
        GsdType type;
        uint64_t N;
        uint32_t M;
        std::vector<char> bytes;
    };
    std::string path_;
    std::string application_, schema_;
    uint32_t schemaVersion_ = 0;
    std::vector<std::string> names_;
    size_t namesWritten_ = 0;                 // names already in the file's namelist
    std::vector<Entry> index_;
    std::vector<Pending> pending_;
    uint64_t frame_ = 0, fileSize_ = 0;
    uint64_t indexLoc_ = 0, indexCap_ = 0, nameLoc_ = 0, nameCap_ = 0;   // nameCap_ in 64-byte units
    void writeHeader(std::FILE *f) const;
};

size_t gsd_type_size(GsdType t);

}  // namespace tild
