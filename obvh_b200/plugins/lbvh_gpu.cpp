// lbvh_gpu.cpp - the "lbvh_gpu" intersector plugin: liblbvh_gpu.so exports the
// one symbol the reference's loader looks up (kr_ads_load, src/common/ads.c:6-32;
// the reference plugin is src/ads/lbvh_gpu/module.c:6-41) and forwards every
// action to the shared core in libobvh_b200.so.
#include "obvh_plugin.h"

extern "C" __attribute__((visibility("default"))) kr_error korangar_ads_action(kr_ads* ads, kr_handle descriptor,
                                                                               kr_ads_action action) {
    return obvh_ads_action(OBVH_ADS_LBVH, ads, descriptor, action);
}
