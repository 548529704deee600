// Instantiations of the J/K launchers for one slice of the classes (one
// file per slice so the build compiles them in parallel).
#include "jk_launch.cuh"

void jk_register_22(JKTables* T) {
    JK_REG(2, 2, 0, 0)
    JK_REG(2, 2, 1, 0)
    JK_REG(2, 2, 1, 1)
    JK_REG(2, 2, 2, 0)
    JK_REG(2, 2, 2, 1)
    JK_REG(2, 2, 2, 2)
}
