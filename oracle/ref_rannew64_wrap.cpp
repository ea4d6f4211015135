// extern "C" wrapper for the reference's rannew64 (rannew64.cu defines it as
// returning double while encabezados.h declares float, so this wrapper lives
// in a translation unit that does not include that header).  Test oracle only.
double rannew64(long *pidum);
extern "C" double ref_rannew64(long *pidum) { return rannew64(pidum); }
