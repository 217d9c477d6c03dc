/* Empty: cooling is compiled out of the hydro pair path. */
