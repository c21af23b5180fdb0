// lucasntt: the reference's command line (main.cpp), over liblucasntt.so.
//
//   lucasntt [exponent [iterations [prefix [fft]]]]
//
// Options come from LucasNTT.ini in the working directory (same keys as the
// reference); results go to <prefix>.dat/.txt/.env or the ini's file names.
// Exit status 1 with a message on any error, as main.cpp:22-36.
#include <cstdio>
#include <stdexcept>

#include "main_process.h"

int main(int argc, char** argv) {
  try {
    lucasntt::MainProcess main_process(argc, argv);
    main_process.Run();
  } catch (const std::runtime_error& e) {
    std::printf("%s\n", e.what());
    return 1;
  } catch (...) {
    std::printf("Unhandled exception! Abort!\n");
    return 1;
  }
  return 0;
}
