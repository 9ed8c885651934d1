// fwt_tube -- the command-line stand-in for the reference program `tube` (tube.f90:30-1240).
// Run it in a directory holding centerline_input.dat and parameters_input.dat; it writes the
// reference's output tree under ./output.  The C++ host replaces the Fortran host because this
// toolchain has no Fortran compiler; fortran/fwt_iface.f90 is the iso_c_binding module a
// Fortran host would use instead.
//
//   fwt_tube [rundir] [--fp64] [--walk] [--device K] [--u-out] [--d-out]
//
// --u-out / --d-out also write field_uw.dat / field_wd.dat (the reference's compile-time
// switches u_out and d_out, tube.f90:55).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "fwt.h"

int main(int argc, char **argv)
{
    std::string dir = ".";
    fwt_params p;
    fwt_default_params(&p);
    int u_out = 0, d_out = 0;
    for (int i = 1; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--fp64")) p.precision = 64;
        else if (!std::strcmp(argv[i], "--walk")) p.deposit_mode = 1;
        else if (!std::strcmp(argv[i], "--device") && i + 1 < argc) p.device = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--u-out")) u_out = 1;
        else if (!std::strcmp(argv[i], "--d-out")) d_out = 1;
        else dir = argv[i];
    }
    int rc;
    if (!u_out && !d_out) {
        rc = fwt_run_dir(dir.c_str(), &p);
    } else {
        // fwt_run_dir's steps with the optional outputs switched on
        fwt_ctx *h = nullptr;
        rc = fwt_create(&p, &h);
        if (rc == 0) rc = fwt_load_inputs(h, (dir + "/centerline_input.dat").c_str(), (dir + "/parameters_input.dat").c_str());
        if (rc == 0) rc = fwt_set_outputs(h, u_out, d_out);
        if (rc == 0) rc = fwt_run(h);
        if (rc == 0) rc = fwt_write_outputs(h, (dir + "/output").c_str());
        if (h) fwt_destroy(h);
    }
    if (rc) {
        char msg[512];
        fwt_last_error(msg, sizeof msg);
        std::fprintf(stderr, "fwt_tube: error %d: %s\n", rc, msg);
        return 1;
    }
    std::printf("fwt_tube: outputs written to %s/output\n", dir.c_str());
    return 0;
}
