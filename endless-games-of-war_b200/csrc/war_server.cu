// war_server.cu — continuous-batching job server (placeholder until the serving loop lands).
#include "war_host.h"

using namespace war;

extern "C" {
int war_server_create(const war_server_cfg*, war_server** out) {
    if (out) *out = nullptr;
    return fail(WAR_EINVAL, "the serving loop is not part of this build yet");
}
int war_server_submit(war_server*, const war_job*, uint64_t*) { return fail(WAR_EINVAL, "no server"); }
int war_server_poll(war_server*, uint64_t, war_result*, war_job_status*) { return fail(WAR_EINVAL, "no server"); }
int war_server_drain(war_server*, double) { return fail(WAR_EINVAL, "no server"); }
int war_server_stats(war_server*, uint64_t*, uint64_t*, uint64_t*) { return fail(WAR_EINVAL, "no server"); }
int war_server_destroy(war_server*) { return WAR_OK; }
}
