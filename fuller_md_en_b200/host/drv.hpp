// drv.hpp -- pieces shared by the fuller_*_gpu drivers: status checks and
// the event schedule of the reference's step loop (LJ:830-936,
// AI:855-950, MM:1174-1274).  Steps between two events run on the device as
// one fmd_system_run call; the host wakes up only at monitor, OVITO and
// restart steps, where the reference reads state too.
#pragma once
#include <cstdio>
#include <cstdlib>
#include <string>

#include "fmd_host.hpp"
#include "fullermd.h"

namespace fmdh {

inline void check(fmd_ctx* ctx, int rc, const char* what) {
    if (rc == FMD_OK) return;
    fprintf(stderr, "Error: %s failed: %s (%s)\n", what, fmd_status_string(rc), ctx ? fmd_ctx_last_error(ctx) : "");
    exit(1);
}

struct Schedule {
    int coldstart = 0, warmup = 0, total = 0;
    int prn = 1, prn_pre = 1;          // monitor cadence after / during cold+warm phases
    int nrec_o = 0, nrec_rst = 0;
    bool ovito = false;

    // LJ:830-834: prn = mon or total/50; warm-up cadence norm/freq/some.
    void set_monitor(int mon_interval, const std::string& warmup_mon_mode) {
        prn = mon_interval > 0 ? mon_interval : std::max(1, total / 50);
        prn_pre = prn;
        if (coldstart + warmup > 0) {
            int div = 100;
            if (warmup_mon_mode == "freq") div = 10;
            else if (warmup_mon_mode == "some") div = 1000;
            prn_pre = std::max(1, (coldstart + warmup) / div);
        }
    }
    int cur_prn(int g) const { return g <= coldstart + warmup ? prn_pre : prn; }
    bool monitor(int g) const { return g % cur_prn(g) == 0 || g == total; }
    bool ovito_at(int g) const { return ovito && g % nrec_o == 0; }
    bool restart_at(int g) const { return nrec_rst > 0 && (g % nrec_rst == 0 || g == total); }
    bool event(int g) const { return monitor(g) || ovito_at(g) || restart_at(g); }
    int next_event(int g) const {
        while (g < total && !event(g)) g++;
        return g;
    }
    const char* phase(int g) const { return g <= coldstart ? "COLD" : g <= coldstart + warmup ? "WARM" : "PROD"; }
};

// Device name and memory for the banner (replaces acc_get_property, LJ:726-739).
inline void device_banner(int dev) {
    char name[128] = {0};
    double gb = 0;
    if (fmd_device_info(dev, name, sizeof(name), &gb) == FMD_OK) {
        printf("  GPU device      : %d (%s)\n", dev, name);
        printf("  GPU VRAM        : %.2f GB\n", gb);
    }
}

}  // namespace fmdh
