/*
 * Minimal stand-in for <embree4/rtcore.h> (embree itself is absent: external/embree is an
 * empty submodule). Only the types and the four calls the reference's bvh/bvh.h makes
 * inline are provided; BVH's out-of-line members are implemented by oracle/ref/ref_bvh.cpp
 * on the oracle's CPU BVH instead of the reference's bvh/bvh.cpp. Test infrastructure only.
 */
#pragma once
#include <vector>

struct RTCDeviceTy {};
struct RTCSceneTy {
    std::vector<float> verts; /* 9 floats per triangle, insertion order = geomID */
    void *accel = nullptr;    /* orc_bvh* */
};
typedef RTCDeviceTy *RTCDevice;
typedef RTCSceneTy *RTCScene;

inline RTCDevice rtcNewDevice(const char *) { return new RTCDeviceTy; }
inline RTCScene rtcNewScene(RTCDevice) { return new RTCSceneTy; }
void rtcReleaseScene(RTCScene scene);
inline void rtcReleaseDevice(RTCDevice d) { delete d; }
