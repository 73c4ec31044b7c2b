// Shim of BaseProject Platform/Storage/Path.h: a file name.
#ifndef TSR_SHIM_PATH_H
#define TSR_SHIM_PATH_H
#include <string>
#include <vector>
namespace Storage {
class Path {
public:
    Path() {}
    Path(const char *s) : mS(s) {}
    Path(const std::string &s) : mS(s) {}
    static Path extendLeafName(const Path &p, const char *ending) { return Path(p.mS + ending); }
    static Path extendLeafName(const Path &p, const std::string &ending) { return Path(p.mS + ending); }
    const std::string &getString() const { return mS; }
    const char *getCString() const { return mS.c_str(); }
private:
    std::string mS;
};
}  // namespace Storage
#endif
