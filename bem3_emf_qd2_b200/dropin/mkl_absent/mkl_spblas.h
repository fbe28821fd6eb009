/* Empty: with the solver replaced by libbem3qd2 no remaining source of the program uses MKL;
 * d3qd2_const.h still includes this header, so an empty one stands in where MKL is absent. */
