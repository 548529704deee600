// Instantiations of the J/K launchers (one file per slice of classes so
// the build compiles them in parallel).
#include "jk_launch.cuh"

void jk_register_l1(jk_launch_fn* tab64, jk_launch_fn* tab32) {
    JK_REG(1, 0, 0, 0)
    JK_REG(1, 0, 1, 0)
    JK_REG(1, 0, 1, 1)
    JK_REG(1, 1, 0, 0)
    JK_REG(1, 1, 1, 0)
    JK_REG(1, 1, 1, 1)
}
