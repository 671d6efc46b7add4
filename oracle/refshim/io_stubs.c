/*
 * PLAPACK's out-of-core objects call PLA_Read/PLA_Write from IO/ (not built
 * into the oracle: out-of-core storage is not on the dense-solve path).
 * Test infrastructure only; reaching either is a harness error.
 */
#include <stdio.h>
#include <stdlib.h>

int PLA_Read(void) {
  fprintf(stderr, "oracle: out-of-core IO is not built\n");
  abort();
}
int PLA_Write(void) {
  fprintf(stderr, "oracle: out-of-core IO is not built\n");
  abort();
}
