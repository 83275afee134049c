// Shim: the elastic material's per-point state (temperature and moisture),
// as elastic.cpp uses it.
#pragma once

class BasicISV {
 public:
  virtual ~BasicISV() {}
};

class ElasticISV : public BasicISV {
 public:
  double getTemperature() const { return temperature; }
  double getMoisture() const { return moisture; }
  void setTemperature(double t) { temperature = t; }
  void setMoisture(double m) { moisture = m; }
  double temperature = 0.0, moisture = 0.0;
};
