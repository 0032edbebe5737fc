// The reference's name for the tree header; the tree class is in AIFMMTree.hpp.
#include "AIFMMTree.hpp"
