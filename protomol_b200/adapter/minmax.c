/* ProtoMol's base/fft.c calls min()/max() without declaring them. */
int min(int a, int b) { return a < b ? a : b; }
int max(int a, int b) { return a > b ? a : b; }
