// Shim of BaseProject Platform/Utilities/ParametersManager.h: named Real
// parameters (App.cfg's occupancy values), set by oracle/ref_driver.cpp.
#ifndef TSR_SHIM_PARAMETERSMANAGER_H
#define TSR_SHIM_PARAMETERSMANAGER_H
#include <map>
#include <string>
#include "Platform/DataTypes.h"
namespace Utilities {
class ParametersManager {
public:
    static ParametersManager &getSingleton();
    bool get(Real &out, const std::string &name) const {
        auto it = mValues.find(name);
        if (it == mValues.end()) return false;
        out = it->second;
        return true;
    }
    void set(const std::string &name, Real v) { mValues[name] = v; }
private:
    std::map<std::string, Real> mValues;
};
}  // namespace Utilities
#endif
