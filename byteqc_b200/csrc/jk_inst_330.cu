// Instantiations of the J/K launchers for one slice of the classes (one
// file per slice so the build compiles them in parallel).
#include "jk_launch.cuh"

void jk_register_330(jk_launch_fn* tab64, jk_launch_fn* tab32) {
    JK_REG(3, 3, 0, 0)
    (void)tab32;
}
