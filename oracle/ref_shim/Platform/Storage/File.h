// Shim of BaseProject Platform/Storage/File.h: files live in memory (a map
// from name to bytes, defined in oracle/ref_driver.cpp), so that the
// reference's own writers (Nodes/Leaves/DualCells/Occupancy::saveToFile)
// hand their arrays to the driver.  No header is written.
#ifndef TSR_SHIM_FILE_H
#define TSR_SHIM_FILE_H
#include <map>
#include <string>
#include <vector>
#include "Platform/DataTypes.h"
#include "Platform/Storage/Path.h"

namespace Storage {
std::map<std::string, std::vector<char>> &shim_files();

class File {
public:
    enum Mode { OPEN_READING, CREATE_WRITING, APPENDING };
    File(const Path &p, Mode mode, bool /*binary*/, uint32 /*version*/ = 0) : mName(p.getString()), mPos(0) {
        if (mode == CREATE_WRITING) shim_files()[mName].clear();
    }
    uint64 write(const void *src, uint64 elementSize, uint64 count) {
        std::vector<char> &b = shim_files()[mName];
        const char *s = static_cast<const char *>(src);
        b.insert(b.end(), s, s + elementSize * count);
        return count;
    }
    uint64 read(void *dst, uint64 maxBytes, uint64 elementSize, uint64 count) {
        std::vector<char> &b = shim_files()[mName];
        uint64 n = count;
        if (elementSize * n > maxBytes) n = maxBytes / elementSize;
        if (mPos + elementSize * n > b.size()) n = (b.size() - mPos) / elementSize;
        memcpy(dst, b.data() + mPos, elementSize * n);
        mPos += elementSize * n;
        return n;
    }
private:
    std::string mName;
    uint64 mPos;
};
}  // namespace Storage
#endif
