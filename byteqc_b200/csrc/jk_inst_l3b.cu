// Instantiations of the J/K launchers (one file per slice of classes so
// the build compiles them in parallel).
#include "jk_launch.cuh"

void jk_register_l3b(jk_launch_fn* tab64, jk_launch_fn* tab32) {
    JK_REG(3, 0, 2, 0)
    JK_REG(3, 0, 2, 1)
    JK_REG(3, 0, 2, 2)
    JK_REG(3, 0, 3, 0)
    JK_REG(3, 0, 3, 1)
    JK_REG(3, 0, 3, 2)
    JK_REG(3, 0, 3, 3)
    JK_REG(3, 1, 2, 0)
    JK_REG(3, 1, 2, 1)
    JK_REG(3, 1, 2, 2)
    JK_REG(3, 1, 3, 0)
    JK_REG(3, 1, 3, 1)
    JK_REG(3, 1, 3, 2)
    JK_REG(3, 1, 3, 3)
    JK_REG(3, 2, 2, 0)
    JK_REG(3, 2, 2, 1)
    JK_REG(3, 2, 2, 2)
    JK_REG(3, 2, 3, 0)
    JK_REG(3, 2, 3, 1)
    JK_REG(3, 2, 3, 2)
    JK_REG(3, 2, 3, 3)
    JK_REG(3, 3, 2, 0)
    JK_REG(3, 3, 2, 1)
    JK_REG(3, 3, 2, 2)
    JK_REG(3, 3, 3, 0)
    JK_REG(3, 3, 3, 1)
    JK_REG(3, 3, 3, 2)
    JK_REG(3, 3, 3, 3)
}
