"""Scene file formats upstream of IndexedMesh: Wavefront OBJ (+ MTL) and
the Roxy Binary (RXB) mesh archive."""
