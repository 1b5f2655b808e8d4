// A module with the B200 provider's file name but without its entry point. Test infrastructure.
extern "C" __attribute__((visibility("default"))) int syclfft_b200_unrelated_symbol(void) { return 0; }
