// Instantiations of the J/K launchers for one slice of the classes (one
// file per slice so the build compiles them in parallel).
#include "jk_launch.cuh"

void jk_register_323(JKTables* T) {
    JK_REG(3, 2, 3, 0)
    JK_REG(3, 2, 3, 1)
    JK_REG(3, 2, 3, 2)
    JK_REG(3, 2, 3, 3)
}
