// Shim of BaseProject Platform/FailureHandling/FileCorruptionException.h.
#ifndef TSR_SHIM_FILECORRUPTIONEXCEPTION_H
#define TSR_SHIM_FILECORRUPTIONEXCEPTION_H
#include "Platform/FailureHandling/Exception.h"
#include "Platform/Storage/Path.h"
namespace FailureHandling {
class FileCorruptionException : public Exception {
public:
    FileCorruptionException(const std::string &m, const Storage::Path &p) : Exception(m + ": " + p.getString()) {}
};
}  // namespace FailureHandling
#endif
