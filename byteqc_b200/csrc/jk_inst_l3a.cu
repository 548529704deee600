// Instantiations of the J/K launchers (one file per slice of classes so
// the build compiles them in parallel).
#include "jk_launch.cuh"

void jk_register_l3a(jk_launch_fn* tab64, jk_launch_fn* tab32) {
    JK_REG(3, 0, 0, 0)
    JK_REG(3, 0, 1, 0)
    JK_REG(3, 0, 1, 1)
    JK_REG(3, 1, 0, 0)
    JK_REG(3, 1, 1, 0)
    JK_REG(3, 1, 1, 1)
    JK_REG(3, 2, 0, 0)
    JK_REG(3, 2, 1, 0)
    JK_REG(3, 2, 1, 1)
    JK_REG(3, 3, 0, 0)
    JK_REG(3, 3, 1, 0)
    JK_REG(3, 3, 1, 1)
}
