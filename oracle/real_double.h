/* Forces the reference's REAL to double without editing it.
 *
 * include/type.h guards itself with TYPE_H and symbolic.h includes it by quoted path, so an
 * include-path override cannot replace it; pre-including this file (gcc -include) defines the
 * guard first, which turns the reference's `typedef float REAL` (include/type.h:3) into a no-op.
 * Test infrastructure only: used when compiling the reference sources into oracle/_ref/.
 */
#ifndef TYPE_H
#define TYPE_H
typedef double REAL;
#endif
