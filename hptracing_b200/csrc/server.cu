// Serving loop and autotuner (filled in below the render path).
#include "../../include/hpt.h"
#include "engine.h"

using namespace hpt;

struct hpt_server {
  int dummy;
};

extern "C" {

hpt_status hpt_server_create(const hpt_server_config*, hpt_server** out) {
  if (out) *out = nullptr;
  return fail(HPT_ERR_UNSUPPORTED, "server not built yet");
}
hpt_status hpt_server_add_scene(hpt_server*, hpt_scene*, int32_t*) {
  return fail(HPT_ERR_UNSUPPORTED, "server not built yet");
}
hpt_status hpt_server_submit(hpt_server*, int32_t, const hpt_camera*, const hpt_render_params*,
                             uint64_t*) {
  return fail(HPT_ERR_UNSUPPORTED, "server not built yet");
}
hpt_status hpt_server_pump(hpt_server*, int32_t) { return fail(HPT_ERR_UNSUPPORTED, "server not built yet"); }
hpt_status hpt_server_poll(hpt_server*, uint64_t, hpt_request_info*, uint8_t*, float*) {
  return fail(HPT_ERR_UNSUPPORTED, "server not built yet");
}
hpt_status hpt_server_cancel(hpt_server*, uint64_t) { return fail(HPT_ERR_UNSUPPORTED, "server not built yet"); }
int32_t hpt_server_pending(const hpt_server*) { return 0; }
void hpt_server_destroy(hpt_server* s) { delete s; }
hpt_status hpt_autotune(hpt_scene*, const hpt_camera*, const hpt_render_params*, const char*,
                        hpt_tuning*) {
  return fail(HPT_ERR_UNSUPPORTED, "autotune not built yet");
}
}
