// atrbvh_gpu.cpp - the "atrbvh_gpu" intersector plugin: libatrbvh_gpu.so
// exports korangar_ads_action (the reference plugin is
// src/ads/atrbvh_gpu/module.c:6-41) and forwards every action to the shared
// core in libobvh_b200.so.
#include "obvh_plugin.h"

extern "C" __attribute__((visibility("default"))) kr_error korangar_ads_action(kr_ads* ads, kr_handle descriptor,
                                                                               kr_ads_action action) {
    return obvh_ads_action(OBVH_ADS_ATRBVH, ads, descriptor, action);
}
