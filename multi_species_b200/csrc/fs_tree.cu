// Barycentric Lagrange treecode (placeholder until the device treecode lands).
#include "fs_device.cuh"

namespace fsb {

FieldEngine* make_treecode(double, double, double, int, int, bool) {
    fail(FS_ERR_UNSUPPORTED, "treecode field not built yet");
}

}  // namespace fsb
