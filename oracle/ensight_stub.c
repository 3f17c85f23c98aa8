/*
 * ensight_stub.c -- empty stand-ins for the reference's EnSight and legacy
 * VTK field writers and readers, which the partitioner links but does not
 * call (it writes processor<pid>/lattice/* only).  TEST INFRASTRUCTURE ONLY:
 * used by the oracle/Makefile target `partition`.
 */
void readLbeFieldFromEnsight(void) {}
void readScalarFromEnsight(void) {}
void readVectorFromEnsight(void) {}
void updateCaseFile(void) {}
void writeLbeFieldToEnsight(void) {}
void writeMeshToEnsight(void) {}
void writePdfToVTK(void) {}
void writeScalarToEnsight(void) {}
void writeVectorToEnsight(void) {}
void writeVectorToVTK(void) {}
