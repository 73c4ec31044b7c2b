// Shim of BaseProject Platform/FailureHandling/Exception.h.
#ifndef TSR_SHIM_EXCEPTION_H
#define TSR_SHIM_EXCEPTION_H
#include <stdexcept>
#include <string>
namespace FailureHandling {
class Exception : public std::runtime_error {
public:
    explicit Exception(const std::string &m) : std::runtime_error(m) {}
};
}  // namespace FailureHandling
#endif
