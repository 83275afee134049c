// Shim: the reference's console progress indicator (no output here).
#pragma once
class ProgressIndicator {
 public:
  void start(const char*) {}
  void notifyPercentDone(float) {}
  void done() {}
};
