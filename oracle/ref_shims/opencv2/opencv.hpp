/*
 * Build shim: the reference's morphutils.h names a few OpenCV types in
 * declarations that TaiChi.cu never calls.  These empty stand-ins let
 * TaiChi.cu compile; the morphology itself (getSdf) is supplied by
 * oracle/ref_bridge.cpp.  Test infrastructure only.
 */
#pragma once
namespace cv {
struct Mat {};
struct Point { int x, y; };
typedef const Mat &InputArray;
typedef Mat &OutputArray;
}
