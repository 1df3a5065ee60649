// host_idp.cpp - IDP2 / UnionDP drivers (placeholder until the drivers land).
#include "host_idp.h"

namespace gqb {

QueryTreeC *run_idp(int algorithm, GpuqoPlannerInfoC *info) {
    (void)algorithm;
    (void)info;
    set_error(GPUQO_B200_ERR_UNSUPPORTED, "IDP drivers are not built yet");
    return nullptr;
}

}  // namespace gqb
