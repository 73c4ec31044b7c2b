// Shim of BaseProject Platform/Utilities/Array.h: the two helpers the tree
// build calls -- reorder (target[targetIndices[i]] = source[i]) and an
// exclusive (or inclusive) prefix sum.
#ifndef TSR_SHIM_ARRAY_H
#define TSR_SHIM_ARRAY_H
#include <vector>
#include "Platform/DataTypes.h"
namespace Utilities {
template <class T>
class Array {
public:
    static void reorder(T *target, const T *source, const uint32 *targetIndices, const uint64 count) {
        for (uint64 i = 0; i < count; ++i) target[targetIndices[i]] = source[i];
    }
    static void reorder(std::vector<T> &data, const uint32 *targetIndices, const uint32 elementsPerItem = 1) {
        std::vector<T> out(data.size());
        const uint64 items = data.size() / elementsPerItem;
        for (uint64 i = 0; i < items; ++i)
            for (uint32 k = 0; k < elementsPerItem; ++k)
                out[(uint64)targetIndices[i] * elementsPerItem + k] = data[i * elementsPerItem + k];
        data.swap(out);
    }
    static void prefixSum(T *out, const T *in, const uint64 count, const bool inclusive) {
        T s = T();
        for (uint64 i = 0; i < count; ++i) {
            if (inclusive) { s += in[i]; out[i] = s; }
            else { out[i] = s; s += in[i]; }
        }
    }
};
}  // namespace Utilities
#endif
