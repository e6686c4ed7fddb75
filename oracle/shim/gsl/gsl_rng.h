/* Empty stand-in: the reference AM path includes this GSL header but uses nothing from it. */
