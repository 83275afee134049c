// Shim: Node as node.cpp defines it (the reference ships no headers): a
// mesh node's coordinates, numbers and dof count / first dof, the per-node
// text and binary records, and setNumDofPerNode, which numbers the dofs.
// NodeGroup is a plain indexed array of nodes here.
#pragma once
#include <cstdio>
#include <iostream>
#include <vector>

typedef double Coordinate;
struct Point {
  Coordinate x = 0.0, y = 0.0, z = 0.0;
};
enum CoordinateReadOption { X, XY, YZ, XYZ };

template <class T>
class NodeArray {
 public:
  explicit NodeArray(int n = 0) : v_(n) {}
  T& operator[](int i) { return v_[i]; }
  int getNumElements() const { return (int)v_.size(); }

 private:
  std::vector<T> v_;
};

class Node;
typedef NodeArray<Node> NodeGroup;

class Node {
 public:
  Node();
  Node(const Point& n);
  Node(const int NodeNum, const double X, const double Y, const double Z);
  ~Node();
  void Initialize();
  static void readAllNodalCoordinates(Node* node, int numNodes, int numDims, std::istream* inputStream);
  bool read(std::istream& istrm, CoordinateReadOption readOption);
  void readBinary(FILE* fp);
  void writeBinary(FILE* fp);
  void print(std::ostream& ostrm);
  void write(std::ostream& ostrm, int numDims);
  void writeNodeInfo(std::ostream& ostrm, int numDims);
  static void setNumDofPerNode(std::istream* inStream, std::ostream* out, int numNodes, NodeGroup* node,
                               int& totalNumDof);
  void setNumDof(int n) { numDof = n; }
  int getNumDof() const { return numDof; }
  void setFirstDof(int f) { firstDof = f; }
  int getFirstDof() const { return firstDof; }

  Coordinate x, y, z;
  int nodeNum, newNodeNum, firstDof, numDof, numElementsAtNode;
  int* eList;
  bool isActive, isSelected, isMidNode, isFiber;
};
std::ostream& operator<<(std::ostream& o, const Node& node);
