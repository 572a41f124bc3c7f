// dropin_main.cpp - checker for the C++ drop-in (include/hpt_trace_runner.hpp)
// against the reference's own types. Test infrastructure: built by
// oracle/build.py into oracle/_ref/ together with the reference's scene
// sources (src/hp/scene/*.cpp, src/hp/common.cpp, tinyobjloader) and the
// refshim/ stand-ins for Eigen and the OpenCL value types, and linked
// against libhpt.so.
//
// It does what the reference's headless CLI does (src/hptracing.cpp:236-296)
// with its real hp::KDTree and cl_float3:
//     auto scene = std::make_unique<hp::KDTree>(input, mtl_basepath);
//     runner = std::make_unique<hp::TraceRunner>(scene);
//     runner->run(pixels, view_point, up_dir, right_dir,
//                 float(width) / float(height) * angle, angle, width, height,
//                 supersample ? 2 : 1, supersample ? 2 : 1, background_color,
//                 sample, depth, no_diffuse ? 1 : 0, brightness);
// and writes the RGBA8 pixels (width * height * 4 bytes, the rows as run()
// returns them) to the output file.
//
// usage: dropin_runner in.obj out.rgba view up right width height angle
//                      sample depth brightness supersample(0/1)
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <string>
#include <vector>

#include "hp/scene/kdtree.h"
#include "hpt_trace_runner.hpp"

namespace {

cl_float3 parse3(const char* s) {  // str2float3, hptracing.cpp:31-39
  cl_float3 r;
  std::string str(s);
  for (int i = 0; i < 3; ++i) {
    r.s[i] = (float)atof(str.c_str());
    if (i < 2) str = str.substr(str.find(',') + 1);
  }
  r.s[3] = 0.f;
  return r;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 13) {
    fprintf(stderr,
            "usage: %s in.obj out.rgba view up right width height angle sample depth "
            "brightness supersample\n",
            argv[0]);
    return 2;
  }
  hp::g_log_enable = false;
  const std::string input = argv[1];
  std::string mtl_basepath;
  const size_t pos = input.rfind('/');
  if (pos != std::string::npos && pos > 0) mtl_basepath = input.substr(0, pos + 1);
  const cl_float3 view_point = parse3(argv[3]), up_dir = parse3(argv[4]),
                  right_dir = parse3(argv[5]);
  const int width = atoi(argv[6]), height = atoi(argv[7]);
  const float angle = (float)atof(argv[8]);
  const int sample = atoi(argv[9]), depth = atoi(argv[10]);
  const float brightness = (float)atof(argv[11]);
  const bool supersample = atoi(argv[12]) != 0;
  cl_float3 background_color = parse3("0,0,0");

  auto scene = std::make_unique<hp::KDTree>(input, mtl_basepath);
  std::unique_ptr<hp::TraceRunner> runner;
  std::vector<unsigned char> pixels((size_t)width * height * 4);
  try {
    runner = std::make_unique<hp::TraceRunner>(scene);
    runner->run(pixels.data(), view_point, up_dir, right_dir,
                float(width) / float(height) * angle, angle, width, height,
                supersample ? 2 : 1, supersample ? 2 : 1, background_color, sample, depth, 0,
                brightness);
  } catch (hpt::Error& err) {
    fprintf(stderr, "drop-in error %d: %s\n", (int)err.status, err.what());
    return 1;
  }
  FILE* f = fopen(argv[2], "wb");
  if (!f || fwrite(pixels.data(), 1, pixels.size(), f) != pixels.size()) {
    fprintf(stderr, "cannot write %s\n", argv[2]);
    return 1;
  }
  fclose(f);
  hpt_render_stats st;
  hpt_render_stats_get(runner->handle(), &st);
  printf("queries %lld ms %.3f\n", (long long)st.intersect_queries, st.ms_total);
  return 0;
}
