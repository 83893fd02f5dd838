/* Drop-in header: QuaC programs include petscksp.h; everything this engine
 * provides is declared in quac_b200.h. */
#include "../quac_b200.h"
